"""The search that allocates nothing, against the allocating one.

rme_search_given_noalloc serves callers that may not allocate device memory
themselves or through the library — a plugin inside a media pipeline that
owns all of the GPU's memory, or a latency-bound loop that cannot afford
the device-wide synchronisation an allocation brings. They hand over their
own planes, jobs and output buffer. Its results must be exactly those of
rme_frame_search in GIVEN mode on the same jobs, and stay so on the next
call, since its fixed scratch array still holds the previous call's state.

The file name sorts last so that, in a run that stops at the first failure,
every other test has already run.
"""
import ctypes as C

import numpy as np
import pytest

import rivet_h26x_codecs_b200.capi as capi
from _common import assert_results_equal, random_jobs, random_picture, shifted

pytestmark = pytest.mark.gpu


def _caller_planes(ms, pic_id, nplanes, cw):
    """The picture's planes copied into device memory the caller owns."""
    import torch
    planes = [ms.plane(pic_id, k) for k in range(nplanes)]
    rows, cols = planes[0].shape
    host = np.ascontiguousarray(np.stack(planes)).view(np.uint8).ravel()
    buf = torch.zeros(host.nbytes + 16, dtype=torch.uint8, device="cuda")
    buf[:host.nbytes].copy_(torch.from_numpy(host))
    ps = capi.PlaneSet(buf.data_ptr(), rows * cols, cols, (cols - cw) // 2)
    return buf, ps


@pytest.mark.parametrize("codec,bd", [(capi.RME_CODEC_HEVC, 8), (capi.RME_CODEC_H264, 8), (capi.RME_CODEC_HEVC, 10)])
def test_no_alloc_search_equals_the_allocating_one(ms, codec, bd):
    import torch
    rng = np.random.default_rng(2024 + codec * 10 + bd)
    w, h = 160, 96
    ref0 = random_picture(rng, w, h, bd)
    ref1 = shifted(ref0, 3, -2, rng, 1.0)
    src = shifted(ref0, -5, 4, rng, 1.0)
    base = 700 + 10 * codec + bd
    ms.upload(base, src, codec, bd, as_ref=True)
    ms.upload(base + 1, ref0, codec, bd, as_ref=True)
    ms.upload(base + 2, ref1, codec, bd, as_ref=True)
    p = capi.default_params(codec, 30)
    p.predictor_mode = capi.RME_PRED_GIVEN
    if codec == capi.RME_CODEC_H264:
        jobs = random_jobs(rng, codec, w, h, 2, 200, sizes=((16, 16), (16, 8), (8, 16), (8, 8), (8, 4), (4, 4)))
    else:
        jobs = random_jobs(rng, codec, w, h, 2, 300, spread=300)
    want = ms.search(base, [base + 1, base + 2], p, jobs)

    nplanes = 4 if codec == capi.RME_CODEC_H264 else 16
    cw = -(-w // 16) * 16 if codec == capi.RME_CODEC_H264 else w
    keep = []
    bufs = [_caller_planes(ms, i, nplanes, cw) for i in (base, base + 1, base + 2)]
    keep.extend(b for b, _ in bufs)
    src_ps = bufs[0][1]
    refs = (capi.PlaneSet * 2)(bufs[1][1], bufs[2][1])
    d_jobs = torch.from_numpy(jobs.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(len(jobs) * capi.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d = capi.PictureDesc(codec, bd, w, h, w)
    for call in range(2):
        d_out.zero_()
        torch.cuda.synchronize()
        rc = capi.lib().rme_search_given_noalloc(C.byref(d), C.byref(p), C.byref(src_ps), refs, 2,
                                                 C.c_void_p(d_jobs.data_ptr()), len(jobs),
                                                 C.c_void_p(d_out.data_ptr()), None)
        assert rc == capi.RME_OK, rc
        got = d_out.cpu().numpy().view(capi.RESULT_DTYPE)
        assert_results_equal(got, want, f"no-alloc call {call}")


def test_no_alloc_search_refuses_more_jobs_than_its_scratch_holds(ms):
    d = capi.PictureDesc(capi.RME_CODEC_HEVC, 8, 64, 64, 64)
    p = capi.default_params(capi.RME_CODEC_HEVC, 30)
    p.predictor_mode = capi.RME_PRED_GIVEN
    ps = capi.PlaneSet(16, 208 * 224, 224, 80)
    refs = (capi.PlaneSet * 1)(ps)
    rc = capi.lib().rme_search_given_noalloc(C.byref(d), C.byref(p), C.byref(ps), refs, 1, C.c_void_p(16),
                                             65537, C.c_void_p(16), None)
    assert rc == capi.RME_EINVAL


# Each malformed job the kernel must refuse before reading anything it names:
# (field, value) pairs over a good job, per codec.
_BAD_JOBS = [("ref", 2), ("ref", -1), ("w", 68), ("w", 6), ("h", 0), ("x", 160), ("y", -4), ("x", 152),
             ("nseeds", -1)]


@pytest.mark.parametrize("codec", [capi.RME_CODEC_HEVC, capi.RME_CODEC_H264])
def test_no_alloc_search_refuses_a_malformed_job_and_keeps_the_others(ms, codec):
    """The jobs live in device memory, where the host cannot check them: a
    job naming a reference past the list, a block of a bad size or outside
    the picture, or more seeds than the job holds is refused on the device
    (the call returns RME_EDEVICE, its result slot is left as it was) and
    every other job's result is the allocating search's. The next call,
    with good jobs only, is exact again."""
    import torch
    bd = 8
    rng = np.random.default_rng(77 + codec)
    w, h = 160, 96
    ref0 = random_picture(rng, w, h, bd)
    ref1 = shifted(ref0, 2, 1, rng, 1.0)
    src = shifted(ref0, -3, 2, rng, 1.0)
    base = 760 + 10 * codec
    ms.upload(base, src, codec, bd, as_ref=True)
    ms.upload(base + 1, ref0, codec, bd, as_ref=True)
    ms.upload(base + 2, ref1, codec, bd, as_ref=True)
    p = capi.default_params(codec, 30)
    p.predictor_mode = capi.RME_PRED_GIVEN
    sizes = ((16, 16), (8, 8), (16, 8)) if codec == capi.RME_CODEC_H264 else ((8, 8), (16, 16), (32, 32))
    jobs = random_jobs(rng, codec, w, h, 2, 64, sizes=sizes)
    want = ms.search(base, [base + 1, base + 2], p, jobs)
    nplanes = 4 if codec == capi.RME_CODEC_H264 else 16
    bufs = [_caller_planes(ms, i, nplanes, w) for i in (base, base + 1, base + 2)]
    src_ps = bufs[0][1]
    refs = (capi.PlaneSet * 2)(bufs[1][1], bufs[2][1])
    d = capi.PictureDesc(codec, bd, w, h, w)
    too_many = 9 if codec == capi.RME_CODEC_H264 else capi.RME_MAX_SEEDS + 1
    cases = _BAD_JOBS + [("nseeds", too_many)]
    rsize = capi.RESULT_DTYPE.itemsize
    for k, (field, value) in enumerate(cases):
        bad = jobs.copy()
        i = (7 * k + 3) % len(jobs)
        bad[i][field] = value
        if field == "x" and value == 152:  # inside the picture, but 8 + 16 past its right edge
            bad[i]["w"] = 16
        d_jobs = torch.from_numpy(bad.view(np.uint8).copy()).cuda()
        d_out = torch.full((len(jobs) * rsize,), 0xAB, dtype=torch.uint8, device="cuda")
        rc = capi.lib().rme_search_given_noalloc(C.byref(d), C.byref(p), C.byref(src_ps), refs, 2,
                                                 C.c_void_p(d_jobs.data_ptr()), len(jobs),
                                                 C.c_void_p(d_out.data_ptr()), None)
        assert rc == capi.RME_EDEVICE, (field, value, rc)
        raw = d_out.cpu().numpy()
        assert (raw[i * rsize:(i + 1) * rsize] == 0xAB).all(), f"{field}={value}: the refused job's slot was written"
        got = raw.view(capi.RESULT_DTYPE)
        keep = np.arange(len(jobs)) != i
        assert_results_equal(got[keep], want[keep], f"{field}={value}: the other jobs")
    d_jobs = torch.from_numpy(jobs.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(len(jobs) * rsize, dtype=torch.uint8, device="cuda")
    rc = capi.lib().rme_search_given_noalloc(C.byref(d), C.byref(p), C.byref(src_ps), refs, 2,
                                             C.c_void_p(d_jobs.data_ptr()), len(jobs),
                                             C.c_void_p(d_out.data_ptr()), None)
    assert rc == capi.RME_OK, rc
    assert_results_equal(d_out.cpu().numpy().view(capi.RESULT_DTYPE), want, "good jobs after the refused ones")
