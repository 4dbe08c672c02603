"""The asynchronous search (rme_frame_search_async + rme_sync) against the
synchronous one: an encoder queues picture t+1's search, makes its mode
decision for picture t on the host while the device searches, then syncs.
Every result must equal the synchronous call's (and so the oracle's)."""
import ctypes as C

import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
import rivet_h26x_codecs_b200.synth as synth
from _common import assert_results_equal

HEVC, H264 = capi.RME_CODEC_HEVC, capi.RME_CODEC_H264
pytestmark = pytest.mark.gpu


def _pinned_results(n):
    import torch
    buf = torch.zeros(n * capi.RESULT_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    return buf, buf.numpy().view(capi.RESULT_DTYPE)


def test_pictures_searched_while_the_host_works_equal_the_synchronous_search(ms):
    import torch
    seq = synth.make_sequence(HEVC, 256, 192, 8, 8, 41, 64, 64, 2.0)
    p = oracle.params(HEVC, 32, hevc_search_range=48)
    for i, f in enumerate(seq.frames):
        ms.upload(900 + i, f, HEVC, 8, as_ref=True)
    pics = [(900 + t, [900 + t - 1, 900 + t - 2]) for t in range(2, 8)]
    want = [ms.search(s, r, p) for s, r in pics]
    n = ms.result_count(*pics[0], p)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    bufs = [_pinned_results(n) for _ in pics]
    # Picture t's "mode decision" (here: the oracle's search of it, on the
    # host) runs while picture t+1 is searched on the device.
    ms.search_async(*pics[0], p, bufs[0][1], stream=sh)
    for k in range(len(pics)):
        assert ms.sync(sh) == 0
        assert_results_equal(bufs[k][1], want[k], f"picture {k} after sync")
        if k + 1 < len(pics):
            ms.search_async(*pics[k + 1], p, bufs[k + 1][1], stream=sh)
        t = pics[k][0] - 900
        host = oracle.frame_search(HEVC, 8, seq.frames[t], [seq.frames[t - 1], seq.frames[t - 2]], p)
        assert_results_equal(host, want[k], f"host work on picture {k}")


def test_more_searches_in_flight_than_slots_and_into_device_memory(ms):
    """Six launches queued before one sync (the context keeps four in
    flight: the fifth and sixth wait for the oldest), half of them into
    device memory."""
    import torch
    seq = synth.make_sequence(HEVC, 192, 128, 8, 8, 43, 64, 64, 2.0)
    h264 = synth.make_sequence(H264, 96, 64, 8, 4, 44, 16, 32, 2.0)
    ph = oracle.params(HEVC, 30)
    p4 = oracle.params(H264, 28)
    for i, f in enumerate(seq.frames):
        ms.upload(950 + i, f, HEVC, 8, as_ref=True)
    for i, f in enumerate(h264.frames):
        ms.upload(980 + i, f, H264, 8, as_ref=True)
    pics = [(950 + t, [950 + t - 1], ph) for t in range(1, 5)] + [(980 + t, [980 + t - 1], p4) for t in (1, 2)]
    want = [ms.search(s, r, q) for s, r, q in pics]
    outs = []
    for k, (s, r, q) in enumerate(pics):
        n = ms.result_count(s, r, q)
        if k % 2:
            dev = torch.zeros(n * capi.RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda:0")
            outs.append(dev)
            ms.search_async(s, r, q, dev)
        else:
            buf, view = _pinned_results(n)
            outs.append((buf, view))
            ms.search_async(s, r, q, view)
    assert ms.sync() == 0
    for k, o in enumerate(outs):
        got = o.cpu().numpy().view(capi.RESULT_DTYPE) if hasattr(o, "data_ptr") else o[1]
        assert_results_equal(got, want[k], f"launch {k}")


def test_an_asynchronous_search_refuses_pageable_memory(ms):
    seq = synth.make_sequence(HEVC, 64, 64, 8, 2, 45, 64, 32, 2.0)
    for i, f in enumerate(seq.frames):
        ms.upload(990 + i, f, HEVC, 8, as_ref=True)
    p = oracle.params(HEVC, 30)
    out = np.zeros(ms.result_count(991, [990], p), capi.RESULT_DTYPE)
    f = ms._frame(991, [990])
    rc = capi.lib().rme_frame_search_async(ms.ctx, C.byref(f), C.byref(p),
                                           C.cast(out.ctypes.data, C.POINTER(capi.Result)), None)
    assert rc == capi.RME_EINVAL
    assert ms.sync() == 0
