"""ORACLE — test infrastructure, not product code.

ctypes wrapper of liboracle_me.so (the C++ restatement of the reference's
motion search in this directory). Imported only by tests/, by
__graft_entry__.smoke() as the checker, and by bench.py's CPU legs.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

import rivet_h26x_codecs_b200.capi as capi

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_me.so"

_PD, _PP, _PR, _PJ = (C.POINTER(capi.PictureDesc), C.POINTER(capi.Params), C.POINTER(capi.Result),
                      C.POINTER(capi.Job))
_SIGS = {
    "orc_params_default": (None, [_PP, C.c_int32, C.c_int32]),
    "orc_standalone_blocks": (C.c_int, [_PD, _PP, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "orc_frame_result_count": (C.c_int, [_PD, _PP, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "orc_frame_search": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), _PP, _PJ, C.c_int32,
                                   C.c_int32, _PR]),
    "orc_hevc_bi": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), _PP, C.POINTER(capi.BiJob),
                              C.c_int32, C.c_int32, C.POINTER(C.c_uint32), _PR]),
    "orc_wp_moments": (C.c_int, [_PD, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]),
    "orc_weighted_sad": (C.c_int, [_PD, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                   C.POINTER(C.c_uint64)]),
    "orc_weighted_samples": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                       C.c_int32, C.c_void_p]),
    "orc_h264_bi_refine": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), _PP,
                                     C.POINTER(capi.H264BiJob), C.c_int32, C.c_int32, C.c_int32, C.POINTER(capi.Mv),
                                     C.POINTER(C.c_uint32)]),
    "orc_hevc_weighted_refine": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), _PP, _PJ,
                                           C.c_int32, C.c_int32, C.c_int32, C.c_int32, _PR]),
    "orc_hevc_bi_weighted": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), _PP,
                                       C.POINTER(capi.BiJob), C.c_int32, C.POINTER(C.c_int32),
                                       C.POINTER(C.c_uint32)]),
    "orc_frames_search_mt": (C.c_int, [_PD, C.c_int32, C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p),
                                       _PP, C.c_int32, C.c_int32, _PR, C.POINTER(C.c_int64),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "orc_hevc_decide": (C.c_int, [_PD, _PP, C.c_int32, _PR, C.POINTER(C.c_int32), C.POINTER(C.c_uint8)]),
    "orc_sad": (C.c_uint32, [C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                             C.c_int32]),
    "orc_satd": (C.c_uint32, [C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                              C.c_int32]),
    "orc_h264_lambda": (C.c_float, [C.c_int32]),
    "orc_hevc_lambda": (C.c_float, [C.c_int32, C.c_int32, C.c_float]),
    "orc_h264_cost_table": (None, [C.c_float, C.POINTER(C.c_uint16)]),
    "orc_hevc_mv_bits": (C.c_uint32, [C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "orc_h264_planes": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.c_void_p]),
    "orc_hevc_planes": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_int32)]),
    "orc_h264_qpel_direct": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                       C.c_int32, C.c_int32, C.c_void_p]),
    "orc_hevc_predict": (C.c_int, [_PD, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_int32, C.c_void_p]),
    "orc_chroma_predict": (C.c_int, [_PD, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(capi.Mv), C.c_void_p]),
    "orc_lowres": (C.c_int, [_PD, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p,
                             C.POINTER(C.c_int32)]),
    "orc_lowres_search": (C.c_int, [_PD, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "orc_lowres_bi_cost": (C.c_int, [_PD, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
}

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        h = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def desc(codec: int, pic: np.ndarray, bit_depth: int) -> capi.PictureDesc:
    if pic.strides[1] != pic.itemsize:
        raise ValueError("pictures must be row-major with unit sample stride")
    h, w = pic.shape
    return capi.PictureDesc(codec, bit_depth, w, h, pic.strides[0] // pic.itemsize)


def params(codec: int, qp: int, **kw) -> capi.Params:
    p = capi.Params()
    lib().orc_params_default(C.byref(p), codec, qp)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def result_count(d, p, nref: int, njobs: int = 0) -> int:
    n = C.c_int32()
    rc = lib().orc_frame_result_count(C.byref(d), C.byref(p), nref, njobs, C.byref(n))
    assert rc == 0, rc
    return n.value


def standalone_blocks(d, p) -> np.ndarray:
    n = C.c_int32()
    assert lib().orc_standalone_blocks(C.byref(d), C.byref(p), None, C.byref(n)) == 0
    out = np.zeros((n.value, 4), np.int32)
    assert lib().orc_standalone_blocks(C.byref(d), C.byref(p), out.ctypes.data_as(C.POINTER(C.c_int32)),
                                       C.byref(n)) == 0
    return out


def frame_search(codec: int, bit_depth: int, src: np.ndarray, refs, p, jobs: np.ndarray | None = None,
                 simd: int = 0) -> np.ndarray:
    src = np.ascontiguousarray(src)
    d = desc(codec, src, bit_depth)
    njobs = 0 if jobs is None else len(jobs)
    n = result_count(d, p, len(refs), njobs)
    out = np.zeros(n, capi.RESULT_DTYPE)
    refs = [np.ascontiguousarray(r) for r in refs]
    rp = (C.c_void_p * len(refs))(*[r.ctypes.data for r in refs])
    jp = None if jobs is None else C.cast(jobs.ctypes.data, _PJ)
    rc = lib().orc_frame_search(C.byref(d), src.ctypes.data, len(refs), rp, C.byref(p), jp, njobs, simd,
                                C.cast(out.ctypes.data, _PR))
    if rc != 0:
        raise RuntimeError(f"oracle frame_search rc={rc}")
    return out


def hevc_bi(bit_depth: int, src: np.ndarray, refs, p, jobs: np.ndarray, refine: bool):
    """satd_bi_at per job (refine False: uint32 array) or refine_bi per job
    (refine True: results)."""
    src = np.ascontiguousarray(src)
    d = desc(capi.RME_CODEC_HEVC, src, bit_depth)
    jobs = np.ascontiguousarray(jobs, capi.BI_JOB_DTYPE)
    refs = [np.ascontiguousarray(r) for r in refs]
    rp = (C.c_void_p * len(refs))(*[r.ctypes.data for r in refs])
    satd = np.zeros(len(jobs), np.uint32)
    out = np.zeros(len(jobs), capi.RESULT_DTYPE)
    rc = lib().orc_hevc_bi(C.byref(d), src.ctypes.data, len(refs), rp, C.byref(p),
                           C.cast(jobs.ctypes.data, C.POINTER(capi.BiJob)), len(jobs), int(refine),
                           satd.ctypes.data_as(C.POINTER(C.c_uint32)), C.cast(out.ctypes.data, _PR))
    if rc != 0:
        raise RuntimeError(f"oracle hevc_bi rc={rc}")
    return out if refine else satd


def h264_bi_refine(bit_depth: int, src: np.ndarray, refs, p, jobs: np.ndarray, rounds: int = 2,
                   diamond: bool = False):
    """b_mb's bi_refine per job: (vectors n x 2 x 2, costs)."""
    src = np.ascontiguousarray(src)
    d = desc(capi.RME_CODEC_H264, src, bit_depth)
    jobs = np.ascontiguousarray(jobs, capi.H264_BI_JOB_DTYPE)
    refs = [np.ascontiguousarray(r) for r in refs]
    rp = (C.c_void_p * len(refs))(*[r.ctypes.data for r in refs])
    mv = np.zeros((len(jobs), 2, 2), np.int16)
    cost = np.zeros(len(jobs), np.uint32)
    rc = lib().orc_h264_bi_refine(C.byref(d), src.ctypes.data, len(refs), rp, C.byref(p),
                                  C.cast(jobs.ctypes.data, C.POINTER(capi.H264BiJob)), len(jobs), rounds,
                                  int(diamond), C.cast(mv.ctypes.data, C.POINTER(capi.Mv)),
                                  cost.ctypes.data_as(C.POINTER(C.c_uint32)))
    if rc != 0:
        raise RuntimeError(f"oracle h264_bi_refine rc={rc}")
    return mv, cost


def hevc_bi_weighted(bit_depth: int, src: np.ndarray, refs, p, jobs: np.ndarray, weights) -> np.ndarray:
    """satd_bi_at under explicit weighting (log2_wd, w0, w1, o0, o1)."""
    src = np.ascontiguousarray(src)
    d = desc(capi.RME_CODEC_HEVC, src, bit_depth)
    jobs = np.ascontiguousarray(jobs, capi.BI_JOB_DTYPE)
    refs = [np.ascontiguousarray(r) for r in refs]
    rp = (C.c_void_p * len(refs))(*[r.ctypes.data for r in refs])
    wt = np.ascontiguousarray(weights, np.int32)
    out = np.zeros(len(jobs), np.uint32)
    rc = lib().orc_hevc_bi_weighted(C.byref(d), src.ctypes.data, len(refs), rp, C.byref(p),
                                    C.cast(jobs.ctypes.data, C.POINTER(capi.BiJob)), len(jobs),
                                    wt.ctypes.data_as(C.POINTER(C.c_int32)), out.ctypes.data_as(C.POINTER(C.c_uint32)))
    if rc != 0:
        raise RuntimeError(f"oracle hevc_bi_weighted rc={rc}")
    return out


def hevc_weighted_refine(bit_depth: int, src: np.ndarray, refs, p, jobs: np.ndarray, log2_wd: int, weight: int,
                         offset: int) -> np.ndarray:
    """A weighted list's refine_subpel per GIVEN job (seeds[0] the start)."""
    src = np.ascontiguousarray(src)
    d = desc(capi.RME_CODEC_HEVC, src, bit_depth)
    jobs = np.ascontiguousarray(jobs, capi.JOB_DTYPE)
    refs = [np.ascontiguousarray(r) for r in refs]
    rp = (C.c_void_p * len(refs))(*[r.ctypes.data for r in refs])
    out = np.zeros(len(jobs), capi.RESULT_DTYPE)
    rc = lib().orc_hevc_weighted_refine(C.byref(d), src.ctypes.data, len(refs), rp, C.byref(p),
                                        C.cast(jobs.ctypes.data, _PJ), len(jobs), log2_wd, weight, offset,
                                        C.cast(out.ctypes.data, _PR))
    if rc != 0:
        raise RuntimeError(f"oracle hevc_weighted_refine rc={rc}")
    return out


def wp_moments(codec: int, bit_depth: int, cur: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """(sr, sc, srr, src, sad) of `cur` against `ref` (wp_moments)."""
    cur, ref = np.ascontiguousarray(cur), np.ascontiguousarray(ref)
    d = desc(codec, cur, bit_depth)
    out = np.zeros(5, np.uint64)
    assert lib().orc_wp_moments(C.byref(d), cur.ctypes.data, ref.ctypes.data,
                                out.ctypes.data_as(C.POINTER(C.c_uint64))) == 0
    return out


def weighted_sad(codec: int, bit_depth: int, cur, ref, weight: int, shift: int, offset: int) -> int:
    cur, ref = np.ascontiguousarray(cur), np.ascontiguousarray(ref)
    d = desc(codec, cur, bit_depth)
    out = C.c_uint64()
    assert lib().orc_weighted_sad(C.byref(d), cur.ctypes.data, ref.ctypes.data, weight, shift, offset,
                                  C.byref(out)) == 0
    return out.value


def weighted_samples(codec: int, bit_depth: int, a: np.ndarray, log_wd: int, weight: int, offset: int):
    """The weighted search plane's formula applied to every sample of `a`."""
    a = np.ascontiguousarray(a)
    out = np.empty_like(a)
    rc = lib().orc_weighted_samples(codec, bit_depth, a.ctypes.data, a.size, log_wd, weight, offset, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle weighted_samples rc={rc}")
    return out


def frames_search_mt(codec: int, bit_depth: int, srcs, refs_per_frame, p, simd: int = 1, threads: int = 1):
    """STANDALONE frames on host threads. Returns (results, seconds, plane_seconds)."""
    d = desc(codec, srcs[0], bit_depth)
    nref = len(refs_per_frame[0])
    per = result_count(d, p, nref)
    out = np.zeros(per * len(srcs), capi.RESULT_DTYPE)
    sp = (C.c_void_p * len(srcs))(*[s.ctypes.data for s in srcs])
    flat = [r for rr in refs_per_frame for r in rr]
    rp = (C.c_void_p * len(flat))(*[r.ctypes.data for r in flat])
    offs = np.arange(len(srcs), dtype=np.int64) * per
    secs, psecs = C.c_double(), C.c_double()
    rc = lib().orc_frames_search_mt(C.byref(d), len(srcs), sp, nref, rp, C.byref(p), simd, threads,
                                    C.cast(out.ctypes.data, _PR), offs.ctypes.data_as(C.POINTER(C.c_int64)),
                                    C.byref(secs), C.byref(psecs))
    if rc != 0:
        raise RuntimeError(f"oracle frames_search_mt rc={rc}")
    return out, secs.value, psecs.value


def hevc_decide(d, p, nref: int, res: np.ndarray):
    nb = len(res) // nref
    best = np.zeros(nb, np.int32)
    part = np.zeros((d.height // 8, d.width // 8), np.uint8)
    rc = lib().orc_hevc_decide(C.byref(d), C.byref(p), nref, C.cast(res.ctypes.data, _PR),
                               best.ctypes.data_as(C.POINTER(C.c_int32)), part.ctypes.data_as(C.POINTER(C.c_uint8)))
    assert rc == 0
    return best, part


def sad(bd, a, b, simd=0) -> int:
    h, w = a.shape
    return lib().orc_sad(bd, a.ctypes.data, a.strides[0] // a.itemsize, b.ctypes.data, b.strides[0] // b.itemsize,
                         w, h, simd)


def satd(bd, a, b, simd=0) -> int:
    h, w = a.shape
    return lib().orc_satd(bd, a.ctypes.data, a.strides[0] // a.itemsize, b.ctypes.data, b.strides[0] // b.itemsize,
                          w, h, simd)


def h264_planes(pic: np.ndarray, bit_depth: int, pad: int = 32) -> np.ndarray:
    d = desc(capi.RME_CODEC_H264, pic, bit_depth)
    cw, ch = -(-d.width // 16) * 16, -(-d.height // 16) * 16
    out = np.zeros((4, ch + 2 * pad, cw + 2 * pad), pic.dtype)
    assert lib().orc_h264_planes(C.byref(d), pic.ctypes.data, pad, out.ctypes.data) == 0
    return out


def hevc_planes(pic: np.ndarray, bit_depth: int, pad: int = 80, force_quarter: bool = False, simd: int = 0):
    """The padded plane and its 15 phases (HalfPlanes), interpolated by the
    scalar passes or (simd=1) the AVX2 rung."""
    d = desc(capi.RME_CODEC_HEVC, pic, bit_depth)
    out = np.zeros((16, d.height + 2 * pad, d.width + 2 * pad), pic.dtype)
    ext = C.c_int32()
    flags = int(force_quarter) | (2 if simd else 0)
    assert lib().orc_hevc_planes(C.byref(d), pic.ctypes.data, pad, flags, out.ctypes.data,
                                 C.byref(ext)) == 0
    return out, ext.value


def h264_qpel_direct(pic, bit_depth, xi, yi, xf, yf, w, h, pad=32):
    d = desc(capi.RME_CODEC_H264, pic, bit_depth)
    out = np.zeros((h, w), pic.dtype)
    assert lib().orc_h264_qpel_direct(C.byref(d), pic.ctypes.data, pad, xi, yi, xf, yf, w, h, out.ctypes.data) == 0
    return out


def hevc_predict(pic, bit_depth, x, y, mvx, mvy, w, h, pad=80):
    d = desc(capi.RME_CODEC_HEVC, pic, bit_depth)
    out = np.zeros((h, w), pic.dtype)
    assert lib().orc_hevc_predict(C.byref(d), pic.ctypes.data, pad, x, y, mvx, mvy, w, h, out.ctypes.data) == 0
    return out


def chroma_predict(codec, bit_depth, luma_w, luma_h, cb, cr, blocks: np.ndarray, mvs: np.ndarray) -> np.ndarray:
    d = capi.PictureDesc(codec, bit_depth, luma_w, luma_h, luma_w)
    n = int(sum((b[2] // 2) * (b[3] // 2) * 2 for b in blocks))
    out = np.zeros(n, cb.dtype)
    blocks = np.ascontiguousarray(blocks, np.int32)
    mvs = np.ascontiguousarray(mvs, np.int16)
    rc = lib().orc_chroma_predict(C.byref(d), cb.ctypes.data, cr.ctypes.data, cb.strides[0] // cb.itemsize,
                                  len(blocks), blocks.ctypes.data_as(C.POINTER(C.c_int32)),
                                  C.cast(mvs.ctypes.data, C.POINTER(capi.Mv)), out.ctypes.data)
    assert rc == 0
    return out


def lowres(pic: np.ndarray, bit_depth: int, codec: int = capi.RME_CODEC_HEVC):
    """The lookahead's half-resolution plane (padded) and intra costs:
    HEVC's cutree (8-bit) or H.264's lookahead (the stream's samples)."""
    d = desc(codec, pic, bit_depth)
    stride, rows, n = C.c_int32(), C.c_int32(), C.c_int32()
    assert lib().orc_lowres(C.byref(d), pic.ctypes.data, None, C.byref(stride), C.byref(rows), None, C.byref(n)) == 0
    dt = np.uint16 if (codec == capi.RME_CODEC_H264 and bit_depth > 8) else np.uint8
    plane = np.zeros((rows.value, stride.value), dt)
    intra = np.zeros(n.value, np.uint32)
    assert lib().orc_lowres(C.byref(d), pic.ctypes.data, plane.ctypes.data, None, None, intra.ctypes.data, None) == 0
    return plane, intra


def lowres_search(cur: np.ndarray, ref: np.ndarray, bit_depth: int, codec: int = capi.RME_CODEC_HEVC):
    d = desc(codec, cur, bit_depth)
    n = C.c_int32()
    assert lib().orc_lowres(C.byref(d), cur.ctypes.data, None, None, None, None, C.byref(n)) == 0
    cost, nsad = np.zeros(n.value, np.uint32), np.zeros(n.value, np.uint32)
    mv = np.zeros((n.value, 2), np.int16)
    assert lib().orc_lowres_search(C.byref(d), cur.ctypes.data, ref.ctypes.data, cost.ctypes.data, mv.ctypes.data,
                                   nsad.ctypes.data) == 0
    return cost, mv, nsad


def lowres_bi_cost(cur, r0, mv0, r1, mv1, bit_depth, codec: int = capi.RME_CODEC_HEVC):
    d = desc(codec, cur, bit_depth)
    mv0 = np.ascontiguousarray(mv0, np.int16)
    mv1 = np.ascontiguousarray(mv1, np.int16)
    out = np.zeros(len(mv0), np.uint32)
    assert lib().orc_lowres_bi_cost(C.byref(d), cur.ctypes.data, r0.ctypes.data, mv0.ctypes.data, r1.ctypes.data,
                                    mv1.ctypes.data, out.ctypes.data) == 0
    return out
