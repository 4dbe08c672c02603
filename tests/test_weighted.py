"""Weighted prediction for the search: the weighted search planes (H.264
h264_me.rs:653-672, HEVC h265_me.rs:4275-4293) and the weight fit's passes
(wp_moments, weighted_sad: dsp/distortion.rs:206-252). The oracle's
restatement against numpy on the CPU; the device kernels against the
oracle, sample for sample and sum for sum."""
import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
from _common import random_jobs, random_picture, shifted

H264, HEVC = capi.RME_CODEC_H264, capi.RME_CODEC_HEVC


def _np_weighted(codec, bd, v, log_wd, w, o):
    v = v.astype(np.int64)
    if codec == H264:
        p = ((v * w + (1 << (log_wd - 1))) >> log_wd) + o if log_wd >= 1 else v * w + o
    else:
        p = (((v << (14 - bd)) * w + (1 << (log_wd - 1))) >> log_wd) + o
    return np.clip(p, 0, (1 << bd) - 1)


@pytest.mark.parametrize("codec,bd,log_wd,w,o", [(H264, 8, 5, 40, -7), (H264, 8, 0, 1, 12), (H264, 10, 6, -20, 900),
                                                 (HEVC, 8, 12, 70, 3), (HEVC, 10, 10, 50, -40)])
def test_weighted_plane_formula(codec, bd, log_wd, w, o):
    rng = np.random.default_rng(bd + log_wd)
    a = random_picture(rng, 64, 32, bd)
    got = oracle.weighted_samples(codec, bd, a, log_wd, w, o)
    np.testing.assert_array_equal(got.astype(np.int64), _np_weighted(codec, bd, a, log_wd, w, o))


def test_wp_moments_and_weighted_sad_are_the_sums():
    rng = np.random.default_rng(5)
    cur = random_picture(rng, 70, 46, 10)
    ref = random_picture(rng, 70, 46, 10)
    m = oracle.wp_moments(HEVC, 10, cur, ref)
    r, c = ref.astype(np.int64), cur.astype(np.int64)
    assert list(m) == [r.sum(), c.sum(), (r * r).sum(), (r * c).sum(), np.abs(c - r).sum()]
    for wt, sh, off in [(64, 6, 0), (80, 6, -12), (-5, 0, 300), (3, 1, 0)]:
        rnd = 1 << (sh - 1) if sh >= 1 else 0
        p = np.clip(((r * wt + rnd) >> sh) + off, 0, 1023)
        assert oracle.weighted_sad(HEVC, 10, cur, ref, wt, sh, off) == np.abs(p - c).sum()


_SWEEP_WEIGHTS = (-128, -77, -1, 0, 1, 31, 32, 63, 64, 65, 127, 191, 255)


def _sweep_pictures(bd, w, h, seed):
    """The planes dsp/distortion.rs:394-456 sweeps: random samples (twice),
    rails (each sample 0 or the maximum), and all at the maximum."""
    rng = np.random.default_rng(seed)
    top = (1 << bd) - 1
    dt = np.uint8 if bd == 8 else np.uint16
    for trial in range(4):
        if trial < 2:
            yield trial, random_picture(rng, w, h, bd), random_picture(rng, w, h, bd)
        elif trial == 2:
            yield trial, *(rng.choice([0, top], size=(h, w)).astype(dt) for _ in range(2))
        else:
            yield trial, np.full((h, w), top, dt), np.full((h, w), top, dt)


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_weighted_sad_sweep_is_the_closed_form(bd):
    """The reference's weighted-kernel sweep (every weight either table
    carries, shifts 0..7, offsets at both ends, rails) restated for the
    oracle: each sum equals the closed form clip(((r*w + rnd) >> s) + o)."""
    scale = 4 if bd > 8 else 1
    top = (1 << bd) - 1
    for trial, cur, ref in _sweep_pictures(bd, 33, 17, bd):
        r, c = ref.astype(np.int64), cur.astype(np.int64)
        m = oracle.wp_moments(HEVC, bd, cur, ref)
        assert list(m) == [r.sum(), c.sum(), (r * r).sum(), (r * c).sum(), np.abs(c - r).sum()], trial
        for wt in _SWEEP_WEIGHTS:
            for sh in range(8):
                for off in (-128 * scale, -3, 0, 5, 127 * scale):
                    rnd = 1 << (sh - 1) if sh >= 1 else 0
                    want = np.abs(np.clip(((r * wt + rnd) >> sh) + off, 0, top) - c).sum()
                    assert oracle.weighted_sad(HEVC, bd, cur, ref, wt, sh, off) == want, (trial, wt, sh, off)


@pytest.mark.gpu
@pytest.mark.parametrize("bd", [8, 10, 12])
def test_weighted_sad_sweep_on_the_device(ms, bd):
    """The same sweep through the device passes, sum for sum with the oracle."""
    scale = 4 if bd > 8 else 1
    for trial, cur, ref in _sweep_pictures(bd, 200, 24, bd + 100):
        ms.upload(2200, cur, HEVC, bd, as_ref=False)
        ms.upload(2201, ref, HEVC, bd, as_ref=False)
        np.testing.assert_array_equal(ms.wp_moments(2200, 2201), oracle.wp_moments(HEVC, bd, cur, ref))
        for wt in _SWEEP_WEIGHTS:
            for sh in range(8):
                for off in (-128 * scale, -3, 0, 5, 127 * scale):
                    assert ms.weighted_sad(2200, 2201, wt, sh, off) == \
                        oracle.weighted_sad(HEVC, bd, cur, ref, wt, sh, off), (trial, wt, sh, off)
    ms.release(2200)
    ms.release(2201)


@pytest.mark.gpu
@pytest.mark.parametrize("codec,bd,w,h,log_wd,wt,o", [(H264, 8, 352, 288, 5, 40, -7), (H264, 10, 200, 136, 0, 1, 12),
                                                       (HEVC, 8, 416, 240, 12, 70, 3),
                                                       (HEVC, 10, 192, 128, 10, 50, -40)])
def test_weighted_planes_match_the_oracle(ms, codec, bd, w, h, log_wd, wt, o):
    """The weighted plane 0 over the whole padded area, and the search planes
    built from it (the oracle's planes of the weighted picture)."""
    rng = np.random.default_rng(w + bd)
    pic = random_picture(rng, w, h, bd)
    ms.upload(1500, pic, codec, bd, as_ref=True)
    ms.picture_weighted(1500, 1501, log_wd, wt, o)
    if codec == H264:
        base = oracle.h264_planes(pic, bd)
        want = oracle.h264_planes(oracle.weighted_samples(codec, bd, pic, log_wd, wt, o), bd)
        rows, cols = base.shape[1:]
        np.testing.assert_array_equal(ms.plane(1501, 0), oracle.weighted_samples(codec, bd, base[0], log_wd, wt, o))
        for k in range(1, 4):
            ys = slice(2, rows - 3) if k in (2, 3) else slice(0, rows)
            xs = slice(2, cols - 3) if k in (1, 3) else slice(0, cols)
            np.testing.assert_array_equal(ms.plane(1501, k)[ys, xs], want[k][ys, xs], err_msg=f"plane {k}")
    else:
        base, _ = oracle.hevc_planes(pic, bd)
        np.testing.assert_array_equal(ms.plane(1501, 0), oracle.weighted_samples(codec, bd, base[0], log_wd, wt, o))
        want, ext = oracle.hevc_planes(oracle.weighted_samples(codec, bd, pic, log_wd, wt, o), bd, force_quarter=True)
        sl = (slice(80 - ext, 80 + h + ext), slice(80 - ext, 80 + w + ext))
        for k in range(1, 16):
            np.testing.assert_array_equal(ms.plane(1501, k)[sl], want[k][sl], err_msg=f"phase {k}")
    ms.release(1500)
    ms.release(1501)


@pytest.mark.gpu
def test_search_on_a_weighted_h264_reference(ms):
    """GIVEN H.264 jobs against the weighted plane equal the oracle's search
    with the weighted picture as the reference (what PRef::search scores)."""
    rng = np.random.default_rng(17)
    ref = random_picture(rng, 352, 288, 8)
    src = shifted(ref, 3, -2, rng, 1.5)
    ms.upload(1600, src, H264, 8, as_ref=False)
    ms.upload(1601, ref, H264, 8, as_ref=True)
    ms.picture_weighted(1601, 1602, 6, 72, -9)
    p = oracle.params(H264, 27, predictor_mode=capi.RME_PRED_GIVEN)
    jobs = random_jobs(rng, H264, 352, 288, 1, 150)
    got = ms.search(1600, [1602], p, jobs)
    want = oracle.frame_search(H264, 8, src, [oracle.weighted_samples(H264, 8, ref, 6, 72, -9)], p, jobs)
    assert (got == want).all()
    for i in range(3):
        ms.release(1600 + i)


@pytest.mark.gpu
@pytest.mark.parametrize("bd,w,h", [(8, 1920, 1080), (10, 352, 288)])
def test_wp_moments_and_weighted_sad_on_the_device(ms, bd, w, h):
    rng = np.random.default_rng(w * bd)
    ref = random_picture(rng, w, h, bd)
    cur = shifted(ref, 1, 1, rng, 3.0)
    ms.upload(1700, cur, HEVC, bd, as_ref=False)
    ms.upload(1701, ref, HEVC, bd, as_ref=True)
    np.testing.assert_array_equal(ms.wp_moments(1700, 1701), oracle.wp_moments(HEVC, bd, cur, ref))
    for wt, sh, off in [(64, 6, 0), (80, 6, -12), (-5, 0, 300)]:
        assert ms.weighted_sad(1700, 1701, wt, sh, off) == oracle.weighted_sad(HEVC, bd, cur, ref, wt, sh, off)
    ms.release(1700)
    ms.release(1701)


def _weighted_jobs(rng, w, h, n, given):
    """GIVEN jobs whose first seed is a whole-sample start (from `given`,
    the results of a GIVEN search of the same jobs)."""
    jobs = random_jobs(rng, HEVC, w, h, 2, n)
    if given is not None:
        jobs["seeds"][:, 0, 0] = given["int_mvx"]
        jobs["seeds"][:, 0, 1] = given["int_mvy"]
    jobs["nseeds"] = np.maximum(jobs["nseeds"], 1)
    return jobs


def test_identity_weighting_refines_as_the_default():
    """With log2_wd = denom + 14 - bd, weight = 2^denom, offset 0, the
    weighted prediction is the default one: refining from a GIVEN search's
    whole-sample winner reproduces that search's vector, SATD and cost."""
    rng = np.random.default_rng(23)
    ref = random_picture(rng, 160, 96, 8)
    src = shifted(ref, 3, -2, rng, 1.5)
    p = oracle.params(HEVC, 32, predictor_mode=capi.RME_PRED_GIVEN)
    jobs = _weighted_jobs(rng, 160, 96, 40, None)
    jobs["ref"] = 0
    given = oracle.frame_search(HEVC, 8, src, [ref], p, jobs)
    start = jobs.copy()
    start["seeds"][:, 0, 0] = given["int_mvx"]
    start["seeds"][:, 0, 1] = given["int_mvy"]
    got = oracle.hevc_weighted_refine(8, src, [ref], p, start, 6 + 6, 1 << 6, 0)
    for f in ("mvx", "mvy", "satd", "cost"):
        np.testing.assert_array_equal(got[f], given[f], err_msg=f)


@pytest.mark.gpu
@pytest.mark.parametrize("bd,w,h,log2_wd,wt,o", [(8, 352, 288, 12, 70, 3), (10, 416, 240, 9, -20, 100),
                                                  (8, 200, 136, 6, 64, 0)])
def test_weighted_refine_matches_the_oracle(ms, bd, w, h, log2_wd, wt, o):
    rng = np.random.default_rng(w + log2_wd)
    r0 = random_picture(rng, w, h, bd)
    r1 = shifted(r0, -4, 2, rng, 1.0)
    src = shifted(r0, 3, -1, rng, 2.0)
    ms.upload(2000, src, HEVC, bd, as_ref=False)
    ms.upload(2001, r0, HEVC, bd, as_ref=True)
    ms.upload(2002, r1, HEVC, bd, as_ref=True)
    p = oracle.params(HEVC, 32, predictor_mode=capi.RME_PRED_GIVEN)
    jobs = _weighted_jobs(rng, w, h, 150, None)
    jobs["seeds"][:, 0] = (jobs["seeds"][:, 0] // 4) * 4  # whole-sample starts
    got = ms.hevc_weighted_refine(2000, [2001, 2002], p, jobs, log2_wd, wt, o)
    want = oracle.hevc_weighted_refine(bd, src, [r0, r1], p, jobs, log2_wd, wt, o)
    from _common import assert_results_equal
    assert_results_equal(got, want, "weighted refine_subpel")
    for i in range(3):
        ms.release(2000 + i)


@pytest.mark.gpu
def test_reused_ids_take_new_contents(ms):
    """An id uploaded again: with the same geometry its buffer is refilled,
    with another one it is replaced; a weighted plane written over an id in
    use likewise. Searches afterwards see the new contents only, and the
    pictures' device memory goes when the ids are released."""
    rng = np.random.default_rng(29)
    p = oracle.params(HEVC, 32)
    before = ms.memory_used()
    a, b = random_picture(rng, 192, 128, 8), random_picture(rng, 320, 192, 8)
    ms.upload(2100, a, HEVC, 8, as_ref=True)
    for pic in (random_picture(rng, 192, 128, 8), b):
        src = shifted(pic, 2, -3, rng, 1.0)
        ms.upload(2100, pic, HEVC, 8, as_ref=True)
        ms.upload(2101, src, HEVC, 8, as_ref=False)
        assert (ms.search(2101, [2100], p) == oracle.frame_search(HEVC, 8, src, [pic], p)).all()
    ms.upload(2102, b, HEVC, 8, as_ref=True)
    held = []
    for wt, o in ((70, 3), (50, -6)):
        ms.picture_weighted(2102, 2100, 6, wt, o)
        np.testing.assert_array_equal(ms.plane(2100, 0)[80:80 + 192, 80:80 + 320],
                                      oracle.weighted_samples(HEVC, 8, b, 6, wt, o))
        held.append(ms.memory_used())
    assert held[0] == held[1]
    for i in range(3):
        ms.release(2100 + i)
    assert ms.memory_used() == before
