"""Python host API over librivet_me.so.

`MotionSearch` is the reference's motion-search entry point lifted to the
batched boundary: upload pictures once (references get their search planes
built on the device, as the encoders build `Hpel` / `HalfPlanes` once per
reference picture), then search whole frames — STANDALONE (the library's
own predictor rule) or GIVEN (one job per encoder call, carrying the
predictors and seeds `p_mb` / `pick_pu` would pass) — or batches of frames
in one persistent launch. Every call goes through the C ABI; there is no
CPU path.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import capi


class MotionSearch:
    """One device context (rme_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = capi.lib()
        h = C.c_void_p()
        rc = self._lib.rme_ctx_create(C.byref(h), device)
        if rc != 0:
            raise RuntimeError(f"rme_ctx_create failed ({rc}): no usable CUDA device {device}")
        self.ctx = h
        self._desc = {}

    def close(self) -> None:
        if self.ctx:
            self._lib.rme_ctx_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int) -> None:
        capi.check(rc, self.ctx)

    # ---- pictures ---------------------------------------------------------
    def upload(self, pic_id: int, pic: np.ndarray, codec: int, bit_depth: int, as_ref: bool = True,
               stream: int = 0) -> None:
        pic = np.ascontiguousarray(pic)
        want = np.uint8 if bit_depth == 8 else np.uint16
        if pic.dtype != want:
            raise ValueError(f"{bit_depth}-bit pictures are {np.dtype(want).name}")
        h, w = pic.shape
        d = capi.PictureDesc(codec, bit_depth, w, h, w)
        self._check(self._lib.rme_picture_upload(self.ctx, pic_id, C.byref(d), capi.ptr(pic), int(as_ref),
                                                 C.c_void_p(stream)))
        self._desc[pic_id] = d

    def upload_chroma(self, pic_id: int, cb: np.ndarray, cr: np.ndarray) -> None:
        cb, cr = np.ascontiguousarray(cb), np.ascontiguousarray(cr)
        self._check(self._lib.rme_picture_upload_chroma(self.ctx, pic_id, capi.ptr(cb), capi.ptr(cr),
                                                        cb.shape[1], None))

    def build_planes(self, pic_id: int, stream: int = 0) -> None:
        """Rebuild a resident reference's search planes (asynchronous)."""
        self._check(self._lib.rme_picture_build_planes(self.ctx, pic_id, C.c_void_p(stream)))

    def picture_weighted(self, ref_id: int, dst_id: int, log_wd: int, weight: int, offset: int,
                         stream: int = 0) -> None:
        """`dst_id` := the weighted search plane of reference `ref_id` (the
        picture's codec picks H.264's or HEVC's formula)."""
        self._check(self._lib.rme_picture_weighted(self.ctx, ref_id, dst_id, log_wd, weight, offset,
                                                   C.c_void_p(stream)))
        self._desc[dst_id] = self._desc[ref_id]

    def wp_moments(self, cur_id: int, ref_id: int) -> np.ndarray:
        """(sr, sc, srr, src, sad) of `cur_id` against `ref_id`."""
        out = np.zeros(5, np.uint64)
        self._check(self._lib.rme_wp_moments(self.ctx, cur_id, ref_id, out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                             None))
        return out

    def weighted_sad(self, cur_id: int, ref_id: int, weight: int, shift: int, offset: int) -> int:
        out = C.c_uint64()
        self._check(self._lib.rme_weighted_sad(self.ctx, cur_id, ref_id, weight, shift, offset, C.byref(out), None))
        return out.value

    def release(self, pic_id: int) -> None:
        self._check(self._lib.rme_picture_release(self.ctx, pic_id))
        self._desc.pop(pic_id, None)

    def plane(self, pic_id: int, index: int) -> np.ndarray:
        rows, cols = C.c_int32(), C.c_int32()
        self._check(self._lib.rme_picture_download_plane(self.ctx, pic_id, index, None, C.byref(rows), C.byref(cols)))
        d = self._desc[pic_id]
        out = np.zeros((rows.value, cols.value), np.uint8 if d.bit_depth == 8 else np.uint16)
        self._check(self._lib.rme_picture_download_plane(self.ctx, pic_id, index, capi.ptr(out), C.byref(rows),
                                                         C.byref(cols)))
        return out

    def memory_used(self) -> int:
        b = C.c_uint64()
        self._check(self._lib.rme_memory_used(self.ctx, C.byref(b)))
        return b.value

    # ---- search -----------------------------------------------------------
    @staticmethod
    def _frame(src_id: int, ref_ids: Sequence[int], jobs: np.ndarray | None = None) -> capi.Frame:
        f = capi.Frame()
        f.src_id = src_id
        f.nref = len(ref_ids)
        for i, r in enumerate(ref_ids):
            f.ref_ids[i] = r
        if jobs is not None:
            f.jobs = C.cast(jobs.ctypes.data, C.POINTER(capi.Job))
            f.njobs = len(jobs)
        return f

    def result_count(self, src_id: int, ref_ids: Sequence[int], params: capi.Params,
                     jobs: np.ndarray | None = None) -> int:
        f = self._frame(src_id, ref_ids, jobs)
        n = C.c_int32()
        self._check(self._lib.rme_frame_result_count(self.ctx, C.byref(f), C.byref(params), C.byref(n)))
        return n.value

    def search(self, src_id: int, ref_ids: Sequence[int], params: capi.Params,
               jobs: np.ndarray | None = None, stream: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """One frame; results as a structured array (capi.RESULT_DTYPE):
        `out` when given (a caller's reused result buffer, at least the
        result count long), else a new array."""
        if jobs is not None:
            jobs = np.ascontiguousarray(jobs, capi.JOB_DTYPE)
        f = self._frame(src_id, ref_ids, jobs)
        n = self.result_count(src_id, ref_ids, params, jobs)
        if out is None:
            out = np.zeros(n, capi.RESULT_DTYPE)
        elif out.dtype != capi.RESULT_DTYPE or out.size < n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous RESULT_DTYPE array of at least the result count")
        else:
            out = out[:n]
        self._check(self._lib.rme_frame_search(self.ctx, C.byref(f), C.byref(params),
                                               C.cast(out.ctypes.data, C.POINTER(capi.Result)), C.c_void_p(stream)))
        return out

    def search_async(self, src_id: int, ref_ids: Sequence[int], params: capi.Params, out,
                     jobs: np.ndarray | None = None, stream: int = 0) -> None:
        """Queue one frame's search on `stream` and return at once. `out` is
        pinned host memory (a structured array over a pinned buffer, or a
        pinned tensor) or a device tensor of at least the result count; it
        holds the results after sync(stream)."""
        if jobs is not None:
            jobs = np.ascontiguousarray(jobs, capi.JOB_DTYPE)
        f = self._frame(src_id, ref_ids, jobs)
        addr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        self._check(self._lib.rme_frame_search_async(self.ctx, C.byref(f), C.byref(params),
                                                     C.cast(C.c_void_p(addr), C.POINTER(capi.Result)),
                                                     C.c_void_p(stream)))

    def sync(self, stream: int = 0) -> int:
        """Wait for the asynchronous searches queued on `stream`; raises on a
        failed one. Returns the device status bits (0)."""
        st = C.c_uint32()
        self._check(self._lib.rme_sync(self.ctx, C.c_void_p(stream), C.byref(st)))
        return st.value

    def hevc_weighted_refine(self, src_id: int, ref_ids: Sequence[int], params: capi.Params, jobs: np.ndarray,
                             log2_wd: int, weight: int, offset: int) -> np.ndarray:
        """A weighted list's refine_subpel per GIVEN job (seeds[0] the
        whole-sample start): results as capi.RESULT_DTYPE."""
        jobs = np.ascontiguousarray(jobs, capi.JOB_DTYPE)
        f = self._frame(src_id, ref_ids, jobs)
        out = np.zeros(len(jobs), capi.RESULT_DTYPE)
        self._check(self._lib.rme_hevc_weighted_refine(self.ctx, C.byref(f), C.byref(params), log2_wd, weight, offset,
                                                       C.cast(out.ctypes.data, C.POINTER(capi.Result)), None))
        return out

    def bi_satd(self, src_id: int, ref_ids: Sequence[int], params: capi.Params, jobs: np.ndarray,
                stream: int = 0) -> np.ndarray:
        """satd_bi_at per job (capi.BI_JOB_DTYPE): the SATD of each vector
        pair's bi-prediction."""
        jobs = np.ascontiguousarray(jobs, capi.BI_JOB_DTYPE)
        f = self._frame(src_id, ref_ids)
        out = np.zeros(len(jobs), np.uint32)
        self._check(self._lib.rme_bi_satd(self.ctx, C.byref(f), C.byref(params),
                                          C.cast(jobs.ctypes.data, C.POINTER(capi.BiJob)), len(jobs),
                                          out.ctypes.data_as(C.POINTER(C.c_uint32)), C.c_void_p(stream)))
        return out

    def bi_satd_weighted(self, src_id: int, ref_ids: Sequence[int], params: capi.Params, jobs: np.ndarray,
                         log2_wd: int, w0: int, w1: int, o0: int, o1: int, stream: int = 0) -> np.ndarray:
        """satd_bi_at under explicit weighting per job: weighted_bi of the
        two lists' 14-bit predictions."""
        jobs = np.ascontiguousarray(jobs, capi.BI_JOB_DTYPE)
        f = self._frame(src_id, ref_ids)
        out = np.zeros(len(jobs), np.uint32)
        self._check(self._lib.rme_bi_satd_weighted(self.ctx, C.byref(f), C.byref(params),
                                                   C.cast(jobs.ctypes.data, C.POINTER(capi.BiJob)), len(jobs),
                                                   log2_wd, w0, w1, o0, o1,
                                                   out.ctypes.data_as(C.POINTER(C.c_uint32)), C.c_void_p(stream)))
        return out

    def bi_refine(self, src_id: int, ref_ids: Sequence[int], params: capi.Params, jobs: np.ndarray,
                  stream: int = 0) -> np.ndarray:
        """refine_bi per job: one result per job (capi.RESULT_DTYPE), mv the
        refined vector of the job's list."""
        jobs = np.ascontiguousarray(jobs, capi.BI_JOB_DTYPE)
        f = self._frame(src_id, ref_ids)
        out = np.zeros(len(jobs), capi.RESULT_DTYPE)
        self._check(self._lib.rme_bi_refine(self.ctx, C.byref(f), C.byref(params),
                                            C.cast(jobs.ctypes.data, C.POINTER(capi.BiJob)), len(jobs),
                                            C.cast(out.ctypes.data, C.POINTER(capi.Result)), C.c_void_p(stream)))
        return out

    def h264_bi_refine(self, src_id: int, ref_ids: Sequence[int], params: capi.Params, jobs: np.ndarray,
                       rounds: int = 2, diamond: bool = False, stream: int = 0):
        """b_mb's joint refinement of B pairs (capi.H264_BI_JOB_DTYPE):
        (vectors n x 2 x 2 int16, costs)."""
        jobs = np.ascontiguousarray(jobs, capi.H264_BI_JOB_DTYPE)
        f = self._frame(src_id, ref_ids)
        mv = np.zeros((len(jobs), 2, 2), np.int16)
        cost = np.zeros(len(jobs), np.uint32)
        self._check(self._lib.rme_h264_bi_refine(self.ctx, C.byref(f), C.byref(params),
                                                 C.cast(jobs.ctypes.data, C.POINTER(capi.H264BiJob)), len(jobs),
                                                 rounds, int(diamond), C.cast(mv.ctypes.data, C.POINTER(capi.Mv)),
                                                 cost.ctypes.data_as(C.POINTER(C.c_uint32)), C.c_void_p(stream)))
        return mv, cost

    def search_batch(self, frames: Sequence[tuple[int, Sequence[int]]],
                     params: capi.Params | Sequence[capi.Params], stream: int = 0, out=None) -> list:
        """Many STANDALONE frames (src_id, ref_ids) in one persistent launch.

        `out` is where the results go: None (a new host array), a structured
        array of capi.RESULT_DTYPE, or a tensor (device memory, or pinned
        host memory) of at least 32 bytes per result. Device memory keeps the
        results on the device; pinned memory takes them in one direct copy.
        Returns one view of `out` per frame (tensor views are uint8 bytes).
        """
        n = len(frames)
        if isinstance(params, capi.Params):
            params = [params] * n
        fa = (capi.Frame * n)(*[self._frame(s, r) for s, r in frames])
        pa = (capi.Params * n)(*params)
        counts = [self.result_count(s, r, p) for (s, r), p in zip(frames, params)]
        offs = np.zeros(n, np.int64)
        offs[1:] = np.cumsum(counts)[:-1]
        total = int(sum(counts))
        rsize = capi.RESULT_DTYPE.itemsize
        if out is None:
            out = np.zeros(total, capi.RESULT_DTYPE)
        if hasattr(out, "data_ptr"):
            nbytes = out.numel() * out.element_size()
            if nbytes < total * rsize:
                raise ValueError(f"out holds {nbytes} bytes, the results need {total * rsize}")
            addr = out.data_ptr()
        else:
            if out.dtype != capi.RESULT_DTYPE or out.size < total or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous RESULT_DTYPE array of at least the result count")
            addr = out.ctypes.data
        self._check(self._lib.rme_batch_search(self.ctx, fa, pa, n, C.cast(C.c_void_p(addr), C.POINTER(capi.Result)),
                                               offs.ctypes.data_as(C.POINTER(C.c_int64)), C.c_void_p(stream)))
        if hasattr(out, "data_ptr"):
            import torch
            flat = out.view(-1).view(torch.uint8)
            return [flat[o * rsize:(o + c) * rsize] for o, c in zip(offs, counts)]
        return [out[o:o + c] for o, c in zip(offs, counts)]

    def batch_result_count(self, frames: Sequence[tuple[int, Sequence[int]]],
                           params: capi.Params | Sequence[capi.Params]) -> int:
        """Results a search_batch of these frames returns (all frames)."""
        if isinstance(params, capi.Params):
            params = [params] * len(frames)
        return int(sum(self.result_count(s, r, p) for (s, r), p in zip(frames, params)))

    # ---- lookahead at half resolution --------------------------------------
    def lowres_build(self, pic_id: int) -> None:
        """The picture's half-resolution plane and intra costs (on the device)."""
        self._check(self._lib.rme_lowres_build(self.ctx, pic_id, None))

    def lowres_intra(self, pic_id: int) -> np.ndarray:
        bw, bh = C.c_int32(), C.c_int32()
        self._check(self._lib.rme_lowres_info(self.ctx, pic_id, C.byref(bw), C.byref(bh), None))
        out = np.zeros(bw.value * bh.value, np.uint32)
        self._check(self._lib.rme_lowres_info(self.ctx, pic_id, None, None,
                                              out.ctypes.data_as(C.POINTER(C.c_uint32))))
        return out

    def lowres_search(self, cur_id: int, ref_id: int):
        """(cost, mv (n x 2 int16), nsad) per half-resolution block."""
        bw, bh = C.c_int32(), C.c_int32()
        self._check(self._lib.rme_lowres_info(self.ctx, cur_id, C.byref(bw), C.byref(bh), None))
        n = bw.value * bh.value
        cost, nsad = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        mv = np.zeros((n, 2), np.int16)
        self._check(self._lib.rme_lowres_search(self.ctx, cur_id, ref_id, cost.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                C.cast(mv.ctypes.data, C.POINTER(capi.Mv)),
                                                nsad.ctypes.data_as(C.POINTER(C.c_uint32)), None))
        return cost, mv, nsad

    def lowres_search_batch(self, pairs: Sequence[tuple[int, int]]):
        """lowres_search over many (cur, ref) pairs in one launch: per pair
        (cost, mv, nsad), as lowres_search returns them."""
        bw, bh = C.c_int32(), C.c_int32()
        self._check(self._lib.rme_lowres_info(self.ctx, pairs[0][0], C.byref(bw), C.byref(bh), None))
        n, k = bw.value * bh.value, len(pairs)
        cur = np.array([a for a, _ in pairs], np.int32)
        ref = np.array([b for _, b in pairs], np.int32)
        cost, nsad = np.zeros((k, n), np.uint32), np.zeros((k, n), np.uint32)
        mv = np.zeros((k, n, 2), np.int16)
        self._check(self._lib.rme_lowres_search_batch(
            self.ctx, k, cur.ctypes.data_as(C.POINTER(C.c_int32)), ref.ctypes.data_as(C.POINTER(C.c_int32)),
            cost.ctypes.data_as(C.POINTER(C.c_uint32)), C.cast(mv.ctypes.data, C.POINTER(capi.Mv)),
            nsad.ctypes.data_as(C.POINTER(C.c_uint32)), None))
        return [(cost[i], mv[i], nsad[i]) for i in range(k)]

    def lowres_bi_cost(self, cur_id: int, r0_id: int, mv0: np.ndarray, r1_id: int, mv1: np.ndarray) -> np.ndarray:
        mv0 = np.ascontiguousarray(mv0, np.int16)
        mv1 = np.ascontiguousarray(mv1, np.int16)
        out = np.zeros(len(mv0), np.uint32)
        self._check(self._lib.rme_lowres_bi_cost(self.ctx, cur_id, r0_id, C.cast(mv0.ctypes.data, C.POINTER(capi.Mv)),
                                                 r1_id, C.cast(mv1.ctypes.data, C.POINTER(capi.Mv)),
                                                 out.ctypes.data_as(C.POINTER(C.c_uint32)), None))
        return out

    def stats(self) -> capi.Stats:
        s = capi.Stats()
        self._check(self._lib.rme_last_stats(self.ctx, C.byref(s)))
        return s

    def chroma_predict(self, ref_id: int, blocks: np.ndarray, mvs: np.ndarray) -> np.ndarray:
        d = self._desc[ref_id]
        blocks = np.ascontiguousarray(blocks, np.int32)
        mvs = np.ascontiguousarray(mvs, np.int16)
        n = int(sum((b[2] // 2) * (b[3] // 2) * 2 for b in blocks))
        out = np.zeros(n, np.uint8 if d.bit_depth == 8 else np.uint16)
        self._check(self._lib.rme_chroma_predict(self.ctx, ref_id, len(blocks),
                                                 blocks.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 C.cast(mvs.ctypes.data, C.POINTER(capi.Mv)), capi.ptr(out), None))
        return out


def standalone_blocks(codec: int, width: int, height: int, bit_depth: int, params: capi.Params) -> np.ndarray:
    d = capi.PictureDesc(codec, bit_depth, width, height, width)
    n = C.c_int32()
    capi.check(capi.lib().rme_standalone_blocks(C.byref(d), C.byref(params), None, C.byref(n)))
    out = np.zeros((n.value, 4), np.int32)
    capi.check(capi.lib().rme_standalone_blocks(C.byref(d), C.byref(params),
                                                out.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n)))
    return out


def hevc_decide(width: int, height: int, bit_depth: int, params: capi.Params, nref: int, res: np.ndarray):
    """Chosen reference per block and the 8x8-cell map of chosen PU sizes (log2)."""
    d = capi.PictureDesc(capi.RME_CODEC_HEVC, bit_depth, width, height, width)
    nb = len(res) // nref
    best = np.zeros(nb, np.int32)
    part = np.zeros((height // 8, width // 8), np.uint8)
    capi.check(capi.lib().rme_hevc_decide(C.byref(d), C.byref(params), nref,
                                          C.cast(res.ctypes.data, C.POINTER(capi.Result)),
                                          best.ctypes.data_as(C.POINTER(C.c_int32)),
                                          part.ctypes.data_as(C.POINTER(C.c_uint8))))
    return best, part


def distortion_batch(kind: str, a, a_stride: int, a_off, b, b_stride: int, b_off, w: int, h: int, bit_depth: int,
                     out, stream: int = 0):
    """The batched SadFn / SatdFn: out[i] = sad|satd of the w x h blocks at
    a + a_off[i] and b + b_off[i] (strides in samples). `a`, `b`, the
    offsets (int64) and `out` (32-bit) are device tensors; asynchronous on
    `stream`. Returns `out`."""
    lib = capi.lib()
    fn = lib.rme_sad_batch if kind == "sad" else lib.rme_satd_batch
    n = out.numel()
    rc = fn(C.c_void_p(a.data_ptr()), a_stride, C.c_void_p(a_off.data_ptr()), C.c_void_p(b.data_ptr()), b_stride,
            C.c_void_p(b_off.data_ptr()), w, h, bit_depth, n, C.cast(C.c_void_p(out.data_ptr()), C.POINTER(C.c_uint32)),
            C.c_void_p(stream))
    if rc != 0:
        raise RuntimeError(f"rme_{kind}_batch failed: {rc}")
    return out


class Server:
    """The serving loop (rme_serve_*) on its own context: per-frame ME
    requests of many streams; each stream's reference pictures stay
    resident. `resident=False`: the frames that arrived since the last
    launch go into a launch of their own, up to three launches overlapping
    on the device; `resident=True`: one search kernel stays on the GPU and
    frames join its queue. The context is the server's while it runs."""

    def __init__(self, ms: MotionSearch, hbm_budget_bytes: int, max_frames_per_launch: int = 32,
                 max_streams: int = 256, resident: bool = False):
        self._lib = capi.lib()
        self.ms = ms
        o = capi.ServeOpts(hbm_budget_bytes, max_frames_per_launch, max_streams,
                           capi.RME_SERVE_RESIDENT if resident else capi.RME_SERVE_LAUNCHES, 0)
        h = C.c_void_p()
        capi.check(self._lib.rme_serve_start(ms.ctx, C.byref(o), C.byref(h)))
        self.h = h
        self._streams = {}
        self._out = {}

    def open_stream(self, stream_id: int, codec: int, bit_depth: int, width: int, height: int,
                    params: capi.Params, nref: int) -> int:
        """Admit a stream; returns 0, or RME_EBUSY when the budget is spent."""
        d = capi.PictureDesc(codec, bit_depth, width, height, width)
        rc = self._lib.rme_serve_open_stream(self.h, stream_id, C.byref(d), C.byref(params), nref)
        if rc == 0:
            nb = len(standalone_blocks(codec, width, height, bit_depth, params))
            self._streams[stream_id] = [codec, nb, nref, 0]
        elif rc != capi.RME_EBUSY:
            capi.check(rc)
        return rc

    def result_count(self, stream_id: int) -> int:
        """Results the stream's next submitted frame will have."""
        codec, nb, nref, seen = self._streams[stream_id]
        nr = min(nref, seen)
        return 0 if nr == 0 else nb if codec == capi.RME_CODEC_H264 else nb * nr

    def submit(self, stream_id: int, luma: np.ndarray, out: np.ndarray | None = None) -> int:
        """Queue one frame (copied before return); returns the request id.
        The results land in `out` (a RESULT_DTYPE array of at least
        result_count(stream_id) entries that the caller reuses, as an encoder
        reuses its motion field) or in a new array."""
        codec, nb, nref, seen = self._streams[stream_id]
        nr = min(nref, seen)
        count = self.result_count(stream_id)
        if out is not None:
            if out.dtype != capi.RESULT_DTYPE or out.size < count or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous RESULT_DTYPE array of the frame's result count")
        elif nr:
            out = np.zeros(max(count, 1), capi.RESULT_DTYPE)
        rid = C.c_int64()
        luma = np.ascontiguousarray(luma)
        capi.check(self._lib.rme_serve_submit(self.h, stream_id, capi.ptr(luma),
                                              C.cast(out.ctypes.data, C.POINTER(capi.Result)) if out is not None
                                              else None, C.byref(rid)))
        self._streams[stream_id][3] = seen + 1
        self._out[rid.value] = out[:count] if out is not None else np.zeros(0, capi.RESULT_DTYPE)
        return rid.value

    def poll(self, max_n: int = 4096) -> list[dict]:
        """Completed requests since the last poll: dicts with the request id,
        stream, status, submit and done times (s) and the results."""
        buf = (capi.Completion * max_n)()
        n = C.c_int32()
        capi.check(self._lib.rme_serve_poll(self.h, buf, max_n, C.byref(n)))
        done = []
        for c in buf[:n.value]:
            done.append({"id": c.request_id, "stream": c.stream_id, "status": c.status, "submit_s": c.submit_s,
                         "done_s": c.done_s, "results": self._out.pop(c.request_id)})
        return done

    def close_stream(self, stream_id: int) -> None:
        capi.check(self._lib.rme_serve_close_stream(self.h, stream_id))
        self._streams.pop(stream_id, None)

    def stop(self) -> None:
        if self.h:
            capi.check(self._lib.rme_serve_stop(self.h))
            self.h = None
