"""Failure detection without a GPU fault: every device wait of the library
is bounded (a poll limit with back-off) and reports a timeout in a status
word instead of trapping or spinning on. Here one such wait — the
lookahead wavefront's wait on a block that never completes — is made to run
out on purpose, and the device stays usable: a search right after it still
matches the oracle bit for bit."""
import ctypes as C

import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
from _common import random_picture, shifted

HEVC = capi.RME_CODEC_HEVC


def test_the_probe_refuses_bad_limits():
    st = C.c_uint32(0)
    lib = capi.lib()
    assert lib.rme_probe_wait_timeout(0, 0, C.byref(st), None) == capi.RME_EINVAL
    assert lib.rme_probe_wait_timeout(0, 1 << 23, C.byref(st), None) == capi.RME_EINVAL
    assert lib.rme_probe_wait_timeout(0, 100, None, None) == capi.RME_EINVAL


@pytest.mark.gpu
def test_a_wait_that_runs_out_is_reported_and_the_device_stays_usable(ms):
    lib = capi.lib()
    st, secs = C.c_uint32(0), C.c_double(0.0)
    assert lib.rme_probe_wait_timeout(0, 4000, C.byref(st), C.byref(secs)) == 0
    assert st.value == 1  # the timeout bit (RME_EDEVICE when a search sees it)
    assert 0.0 < secs.value < 1.0
    rng = np.random.default_rng(9)
    ref = random_picture(rng, 128, 96, 8)
    src = shifted(ref, 3, -2, rng, 1.0)
    ms.upload(1900, src, HEVC, 8, as_ref=False)
    ms.upload(1901, ref, HEVC, 8, as_ref=True)
    p = oracle.params(HEVC, 32)
    got = ms.search(1900, [1901], p)
    want = oracle.frame_search(HEVC, 8, src, [ref], p)
    assert (got == want).all()
    ms.release(1900)
    ms.release(1901)
