"""The serving loop, in both modes (a launch per batch of arrivals with
launches overlapping, and the resident engine): per-frame requests of
several streams (two codecs, two bit depths, different sizes) give the same
results when each stream is served alone and when all are in the mix, and
the same as the plain per-frame path; admission refuses streams past the
HBM budget."""
import time

import numpy as np
import pytest

import rivet_h26x_codecs_b200.capi as capi
import rivet_h26x_codecs_b200.host as host
import rivet_h26x_codecs_b200.synth as synth
from _common import assert_results_equal

H264, HEVC = capi.RME_CODEC_H264, capi.RME_CODEC_HEVC
pytestmark = pytest.mark.gpu

STREAMS = [  # id, codec, bit depth, width, height, refs, qp (qp 31: HEVC with AMP units)
    (11, HEVC, 8, 192, 128, 2, 32),
    (12, HEVC, 10, 128, 96, 1, 30),
    (13, H264, 8, 96, 64, 1, 28),
    (14, HEVC, 8, 160, 96, 2, 34),
    (15, HEVC, 8, 128, 96, 2, 31),
]
NFRAMES = 4


def _frames(sid, codec, bd, w, h):
    return synth.make_sequence(codec, w, h, bd, NFRAMES, 1000 + sid, 32, 32, 2.0).frames


def _params(codec, qp):
    """HEVC frames without AMP run in the engine's row form; the qp-31
    stream's AMP units keep the dataflow form."""
    p = capi.default_params(codec, qp)
    if codec == HEVC:
        p.hevc_search_range = 32
        if qp == 31:
            p.hevc_amp = 0b0101
    return p


def _wait(server, n, timeout=60.0):
    got, t0 = [], time.time()
    while len(got) < n:
        got += server.poll()
        if time.time() - t0 > timeout:
            raise TimeoutError(f"{len(got)} of {n} requests completed")
        time.sleep(0.001)
    return got


def _serve(streams, interleave, resident):
    with host.MotionSearch(0) as ms:
        srv = host.Server(ms, hbm_budget_bytes=8 << 30, max_frames_per_launch=8, resident=resident)
        try:
            frames = {}
            for sid, codec, bd, w, h, nref, qp in streams:
                assert srv.open_stream(sid, codec, bd, w, h, _params(codec, qp), nref) == 0
                frames[sid] = _frames(sid, codec, bd, w, h)
            ids = {}
            if interleave:  # every stream's frames submitted back to back
                for t in range(NFRAMES):
                    for s in streams:
                        ids[srv.submit(s[0], frames[s[0]][t])] = (s[0], t)
                done = _wait(srv, len(ids))
            else:  # one request at a time
                done = []
                for s in streams:
                    for t in range(NFRAMES):
                        ids[srv.submit(s[0], frames[s[0]][t])] = (s[0], t)
                        done += _wait(srv, 1)
            out = {}
            for c in done:
                assert c["status"] == 0, c
                assert c["done_s"] >= c["submit_s"]
                out[ids[c["id"]]] = c["results"]
            return out, frames
        finally:
            srv.stop()


@pytest.mark.parametrize("resident", [False, True])
def test_results_are_the_same_alone_and_in_the_mix(resident):
    alone = {}
    for s in STREAMS:
        r, frames = _serve([s], interleave=False, resident=resident)
        alone.update(r)
    mix, frames = _serve(STREAMS, interleave=True, resident=resident)
    assert set(mix) == set(alone)
    for key in sorted(alone):
        assert_results_equal(mix[key], alone[key], f"stream {key[0]} frame {key[1]}")
    # and the plain per-frame path on the same pictures
    with host.MotionSearch(0) as ms:
        for sid, codec, bd, w, h, nref, qp in STREAMS:
            fr = frames[sid]
            for t in range(NFRAMES):
                ms.upload(t, fr[t], codec, bd, as_ref=True)
            for t in range(1, NFRAMES):
                refs = [t - 1 - r for r in range(min(nref, t))]
                want = ms.search(t, refs, _params(codec, qp))
                assert_results_equal(alone[(sid, t)], want, f"stream {sid} frame {t} vs plain")
            assert len(alone[(sid, 0)]) == 0  # the first frame only becomes a reference
            for t in range(NFRAMES):
                ms.release(t)


def test_admission_is_bounded_by_the_budget():
    with host.MotionSearch(0) as ms:
        # A stream holds nref + 4 pictures of 16 padded planes (rows of 128-byte multiples).
        picture = ((1920 + 160 + 127) // 128 * 128) * (1080 + 160) * 16 + 256
        one = picture * (2 + 4)
        srv = host.Server(ms, hbm_budget_bytes=int(one * 1.5), max_frames_per_launch=4)
        try:
            p = _params(HEVC, 32)
            assert srv.open_stream(1, HEVC, 8, 1920, 1080, p, 2) == 0
            assert srv.open_stream(2, HEVC, 8, 1920, 1080, p, 2) == capi.RME_EBUSY
            srv.close_stream(1)
            time.sleep(0.05)
            assert srv.open_stream(2, HEVC, 8, 1920, 1080, p, 2) == 0
        finally:
            srv.stop()


@pytest.mark.parametrize("resident", [False, True])
def test_many_frames_recycle_the_engine_slots_and_survive_idle_periods(resident):
    """300 frames of one stream and 60 of another, submitted in bursts with
    pauses: through the resident engine, more frames than it has frame slots
    (each slot reused with a new generation), and pauses long enough for the
    engine kernel to leave and be launched again; through overlapping
    launches, the launch streams' buffers reused. Every checked frame equals
    the plain per-frame path."""
    streams = [(21, HEVC, 8, 128, 64, 2, 32), (22, H264, 8, 96, 64, 1, 28)]
    counts = {21: 300, 22: 60}
    seqs = {sid: synth.make_sequence(codec, w, h, bd, 8, 2000 + sid, 32, 32, 2.0).frames
            for sid, codec, bd, w, h, _, _ in streams}
    pics = {sid: [seqs[sid][t % 8] if (t // 8) % 2 == 0 else seqs[sid][7 - t % 8] for t in range(counts[sid])]
            for sid in counts}
    with host.MotionSearch(0) as ms:
        srv = host.Server(ms, hbm_budget_bytes=8 << 30, max_frames_per_launch=8, resident=resident)
        got = {}
        try:
            for sid, codec, bd, w, h, nref, qp in streams:
                assert srv.open_stream(sid, codec, bd, w, h, _params(codec, qp), nref) == 0
            ids = {}
            t = {sid: 0 for sid in counts}
            burst = 0
            while any(t[s] < counts[s] for s in counts):
                for _ in range(40):
                    for sid in counts:
                        if t[sid] < counts[sid]:
                            ids[srv.submit(sid, pics[sid][t[sid]])] = (sid, t[sid])
                            t[sid] += 1
                done = _wait(srv, len(ids) - len(got))
                for c in done:
                    assert c["status"] == 0, c
                    got[ids[c["id"]]] = c["results"]
                burst += 1
                if burst % 3 == 0:
                    time.sleep(0.6)  # the engine kernel leaves after a quarter second idle
        finally:
            srv.stop()
        for sid, codec, bd, w, h, nref, qp in streams:
            for k in range(1, counts[sid]):
                if k % 7 and k > 20:  # every seventh frame, and the first twenty, against the plain path
                    continue
                ms.upload(100, pics[sid][k], codec, bd, as_ref=True)
                refs = []
                for r in range(min(nref, k)):
                    ms.upload(101 + r, pics[sid][k - 1 - r], codec, bd, as_ref=True)
                    refs.append(101 + r)
                want = ms.search(100, refs, _params(codec, qp))
                assert_results_equal(got[(sid, k)], want, f"stream {sid} frame {k}")
