"""ctypes binding of librivet_me.so — the C ABI declared in include/rivet_me.h.

The structures below mirror the header field for field. The library is the
CUDA path; there is no fallback: if the shared object is missing the import
of `lib()` raises, so a test or a bench can never pass on a silent CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

RME_OK = 0
RME_EINVAL = -1
RME_ENOMEM = -2
RME_ECUDA = -3
RME_ENOTFOUND = -4
RME_EDEVICE = -5
RME_EBUSY = -6
RME_ENOSYS = -7

RME_CODEC_H264 = 0
RME_CODEC_HEVC = 1
RME_PRED_GIVEN = 0
RME_PRED_STANDALONE = 1
RME_JOB_SCORE_ONLY = 1
RME_MAX_SEEDS = 10
RME_MAX_REFS = 4


class Mv(C.Structure):
    _fields_ = [("x", C.c_int16), ("y", C.c_int16)]


class PictureDesc(C.Structure):
    _fields_ = [("codec", C.c_int32), ("bit_depth", C.c_int32), ("width", C.c_int32),
                ("height", C.c_int32), ("stride", C.c_int32)]


class Params(C.Structure):
    _fields_ = [
        ("codec", C.c_int32), ("qp", C.c_int32), ("predictor_mode", C.c_int32),
        ("h264_range", C.c_int32), ("h264_hpel_iters", C.c_int32), ("h264_qpel_iters", C.c_int32),
        ("h264_umh", C.c_int32), ("h264_qpel_diamond", C.c_int32), ("h264_dia", C.c_int32),
        ("h264_refine_ratio", C.c_float), ("h264_vertical_range", C.c_int32), ("h264_pad", C.c_int32),
        ("hevc_search_range", C.c_int32), ("hevc_search_rings", C.c_int32),
        ("hevc_quarter_cross", C.c_int32), ("hevc_lambda_scale", C.c_float), ("hevc_pad", C.c_int32),
        ("hevc_pu_mask", C.c_int32), ("hevc_amp", C.c_int32),
    ]


class Job(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("w", C.c_int32), ("h", C.c_int32),
                ("ref", C.c_int32), ("nseeds", C.c_int32), ("flags", C.c_int32),
                ("mvp", Mv * 2), ("seeds", Mv * RME_MAX_SEEDS)]


class Result(C.Structure):
    _fields_ = [("mv", Mv), ("ref", C.c_int32), ("cost", C.c_uint32), ("satd", C.c_uint32),
                ("int_mv", Mv), ("int_cost", C.c_uint32), ("n_sad", C.c_uint32),
                ("n_satd", C.c_uint32)]


class BiJob(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("w", C.c_int32), ("h", C.c_int32),
                ("ref", C.c_int32 * 2), ("mv", Mv * 2), ("list", C.c_int32), ("mvp", Mv * 2)]


class H264BiJob(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("w", C.c_int32), ("h", C.c_int32),
                ("ref", C.c_int32 * 2), ("mv", Mv * 2), ("mvp", Mv * 2), ("limit", C.c_uint32)]


class Frame(C.Structure):
    _fields_ = [("src_id", C.c_int32), ("nref", C.c_int32), ("ref_ids", C.c_int32 * RME_MAX_REFS),
                ("jobs", C.POINTER(Job)), ("njobs", C.c_int32)]


class PlaneSet(C.Structure):
    _fields_ = [("base", C.c_void_p), ("plane_elems", C.c_int64), ("stride", C.c_int32), ("pad", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("tasks", C.c_uint64), ("sad_candidates", C.c_uint64),
                ("satd_candidates", C.c_uint64), ("sad_samples", C.c_uint64),
                ("satd_samples", C.c_uint64), ("kernel_ms", C.c_float), ("planes_ms", C.c_float)]


RME_SERVE_LAUNCHES, RME_SERVE_RESIDENT = 0, 1


class ServeOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_frames_per_launch", C.c_int32),
                ("max_streams", C.c_int32), ("mode", C.c_int32), ("reserved", C.c_int32)]


class Completion(C.Structure):
    _fields_ = [("request_id", C.c_int64), ("stream_id", C.c_int32), ("status", C.c_int32),
                ("submit_s", C.c_double), ("done_s", C.c_double), ("nresults", C.c_int32)]


# numpy view of rme_result (same layout) for fast comparisons
RESULT_DTYPE = np.dtype([("mvx", "<i2"), ("mvy", "<i2"), ("ref", "<i4"), ("cost", "<u4"),
                         ("satd", "<u4"), ("int_mvx", "<i2"), ("int_mvy", "<i2"),
                         ("int_cost", "<u4"), ("n_sad", "<u4"), ("n_satd", "<u4")])
assert RESULT_DTYPE.itemsize == C.sizeof(Result)
JOB_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("w", "<i4"), ("h", "<i4"), ("ref", "<i4"),
                      ("nseeds", "<i4"), ("flags", "<i4"), ("mvp", "<i2", (2, 2)),
                      ("seeds", "<i2", (RME_MAX_SEEDS, 2))])
assert JOB_DTYPE.itemsize == C.sizeof(Job)
BI_JOB_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("w", "<i4"), ("h", "<i4"), ("ref", "<i4", (2,)),
                         ("mv", "<i2", (2, 2)), ("list", "<i4"), ("mvp", "<i2", (2, 2))])
assert BI_JOB_DTYPE.itemsize == C.sizeof(BiJob)
H264_BI_JOB_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("w", "<i4"), ("h", "<i4"), ("ref", "<i4", (2,)),
                              ("mv", "<i2", (2, 2)), ("mvp", "<i2", (2, 2)), ("limit", "<u4")])
assert H264_BI_JOB_DTYPE.itemsize == C.sizeof(H264BiJob)

# Every entry point include/rivet_me.h declares, with its ctypes signature.
_vp, _i32, _i64, _u32p = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_uint32)
SIGNATURES = {
    "rme_params_default": (None, [C.POINTER(Params), _i32, _i32]),
    "rme_ctx_create": (C.c_int, [C.POINTER(C.c_void_p), _i32]),
    "rme_ctx_destroy": (None, [_vp]),
    "rme_last_error": (C.c_char_p, [_vp]),
    "rme_picture_upload": (C.c_int, [_vp, _i32, C.POINTER(PictureDesc), _vp, _i32, _vp]),
    "rme_picture_upload_chroma": (C.c_int, [_vp, _i32, _vp, _vp, _i32, _vp]),
    "rme_picture_release": (C.c_int, [_vp, _i32]),
    "rme_picture_build_planes": (C.c_int, [_vp, _i32, _vp]),
    "rme_picture_download_plane": (C.c_int, [_vp, _i32, _i32, _vp, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32)]),
    "rme_memory_used": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "rme_frame_result_count": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params),
                                         C.POINTER(C.c_int32)]),
    "rme_standalone_blocks": (C.c_int, [C.POINTER(PictureDesc), C.POINTER(Params),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "rme_frame_search": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), C.POINTER(Result), _vp]),
    "rme_batch_search": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), _i32, C.POINTER(Result),
                                   C.POINTER(C.c_int64), _vp]),
    "rme_frame_search_async": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), C.POINTER(Result), _vp]),
    "rme_batch_search_async": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), _i32, C.POINTER(Result),
                                         C.POINTER(C.c_int64), _vp]),
    "rme_sync": (C.c_int, [_vp, _vp, C.POINTER(C.c_uint32)]),
    "rme_hevc_decide": (C.c_int, [C.POINTER(PictureDesc), C.POINTER(Params), _i32, C.POINTER(Result),
                                  C.POINTER(C.c_int32), C.POINTER(C.c_uint8)]),
    "rme_last_stats": (C.c_int, [_vp, C.POINTER(Stats)]),
    "rme_picture_weighted": (C.c_int, [_vp, _i32, _i32, _i32, _i32, _i32, _vp]),
    "rme_wp_moments": (C.c_int, [_vp, _i32, _i32, C.POINTER(C.c_uint64), _vp]),
    "rme_weighted_sad": (C.c_int, [_vp, _i32, _i32, _i32, _i32, _i32, C.POINTER(C.c_uint64), _vp]),
    "rme_h264_bi_refine": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), C.POINTER(H264BiJob), _i32, _i32,
                                     _i32, C.POINTER(Mv), _u32p, _vp]),
    "rme_probe_wait_timeout": (C.c_int, [_i32, C.c_uint32, _u32p, C.POINTER(C.c_double)]),
    "rme_hevc_weighted_refine": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), _i32, _i32, _i32,
                                           C.POINTER(Result), _vp]),
    "rme_bi_satd": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), C.POINTER(BiJob), _i32, _u32p, _vp]),
    "rme_bi_satd_weighted": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), C.POINTER(BiJob), _i32, _i32,
                                       _i32, _i32, _i32, _i32, _u32p, _vp]),
    "rme_bi_refine": (C.c_int, [_vp, C.POINTER(Frame), C.POINTER(Params), C.POINTER(BiJob), _i32,
                                C.POINTER(Result), _vp]),
    "rme_chroma_predict": (C.c_int, [_vp, _i32, _i32, C.POINTER(C.c_int32), C.POINTER(Mv), _vp, _vp]),
    "rme_lowres_build": (C.c_int, [_vp, _i32, _vp]),
    "rme_lowres_info": (C.c_int, [_vp, _i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _u32p]),
    "rme_lowres_search": (C.c_int, [_vp, _i32, _i32, _u32p, C.POINTER(Mv), _u32p, _vp]),
    "rme_lowres_search_batch": (C.c_int, [_vp, _i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _u32p,
                                          C.POINTER(Mv), _u32p, _vp]),
    "rme_lowres_bi_cost": (C.c_int, [_vp, _i32, _i32, C.POINTER(Mv), _i32, C.POINTER(Mv), _u32p, _vp]),
    "rme_sad_batch": (C.c_int, [_vp, _i64, _vp, _vp, _i64, _vp, _i32, _i32, _i32, _i32, _u32p, _vp]),
    "rme_satd_batch": (C.c_int, [_vp, _i64, _vp, _vp, _i64, _vp, _i32, _i32, _i32, _i32, _u32p, _vp]),
    "rme_serve_start": (C.c_int, [_vp, C.POINTER(ServeOpts), C.POINTER(C.c_void_p)]),
    "rme_serve_open_stream": (C.c_int, [_vp, _i32, C.POINTER(PictureDesc), C.POINTER(Params), _i32]),
    "rme_serve_submit": (C.c_int, [_vp, _i32, _vp, C.POINTER(Result), C.POINTER(C.c_int64)]),
    "rme_serve_poll": (C.c_int, [_vp, C.POINTER(Completion), _i32, C.POINTER(C.c_int32)]),
    "rme_serve_close_stream": (C.c_int, [_vp, _i32]),
    "rme_serve_stop": (C.c_int, [_vp]),
    "rme_probe_int_peak": (C.c_int, [_i32, C.POINTER(C.c_double)]),
    "rme_search_given_noalloc": (C.c_int, [C.POINTER(PictureDesc), C.POINTER(Params), C.POINTER(PlaneSet),
                                           C.POINTER(PlaneSet), _i32, _vp, _i32, _vp, _vp]),
}

PACKAGE_DIR = Path(__file__).resolve().parent
# RIVET_ME_LIB selects another build of the same library (e.g. a variant
# compiled with other settings); by default the in-tree build is loaded.
LIB_PATH = Path(os.environ.get("RIVET_ME_LIB", PACKAGE_DIR / "librivet_me.so"))

_lib = None


def lib() -> C.CDLL:
    """The loaded CUDA library. Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                               "(the motion search has no CPU fallback)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(rc: int, ctx=None) -> None:
    if rc != RME_OK:
        msg = ""
        if ctx is not None:
            raw = lib().rme_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise RuntimeError(f"librivet_me error {rc}: {msg}")


def default_params(codec: int, qp: int) -> Params:
    p = Params()
    lib().rme_params_default(C.byref(p), codec, qp)
    return p


def ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def os_env_flag(name: str) -> bool:
    return os.environ.get(name, "") not in ("", "0")
