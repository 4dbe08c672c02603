"""HEVC bi-prediction for B units (encode/h265_me.rs): satd_bi_at
(4209-4264) and refine_bi (3933-4014). The oracle's restatement against
closed forms on the CPU; the device kernels against the oracle, job for
job, bit for bit."""
import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
from _common import assert_results_equal, random_picture, shifted

HEVC = capi.RME_CODEC_HEVC


def _satd(a: np.ndarray, b: np.ndarray) -> int:
    """dsp/distortion.rs satd: per 4x4 tile the Hadamard sum, (sum + 1) >> 1."""
    h4 = np.array([[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, -1, 1], [1, -1, 1, -1]])
    d = a.astype(np.int64) - b.astype(np.int64)
    total = 0
    for y in range(0, d.shape[0], 4):
        for x in range(0, d.shape[1], 4):
            t = h4 @ d[y:y + 4, x:x + 4] @ h4.T
            total += (int(np.abs(t).sum()) + 1) >> 1
    return total


def _jobs(rng, w, h, n, nref=2, spread=64, far=0.0):
    """Random bi jobs: blocks of the HEVC unit shapes, quarter-sample vectors
    within `spread`, a fraction `far` of them far outside the picture."""
    sizes = ((8, 8), (16, 16), (32, 32), (64, 64), (16, 8), (8, 16), (32, 16), (16, 32), (64, 32), (32, 64),
             (16, 4), (4, 16), (16, 12), (16, 4), (64, 48), (48, 64), (64, 16), (16, 64), (32, 24), (8, 4))
    jobs = np.zeros(n, capi.BI_JOB_DTYPE)
    for i in range(n):
        bw, bh = sizes[rng.integers(len(sizes))]
        jobs[i]["x"] = rng.integers(0, (w - bw) // 4 + 1) * 4
        jobs[i]["y"] = rng.integers(0, (h - bh) // 4 + 1) * 4
        jobs[i]["w"], jobs[i]["h"] = bw, bh
        jobs[i]["ref"] = rng.integers(nref, size=2)
        s = 1200 if rng.random() < far else spread
        jobs[i]["mv"] = rng.integers(-s, s + 1, size=(2, 2))
        jobs[i]["list"] = rng.integers(2)
        jobs[i]["mvp"] = rng.integers(-spread, spread + 1, size=(2, 2))
    return jobs


def test_bi_satd_of_whole_sample_vectors_is_the_rounded_average():
    rng = np.random.default_rng(1)
    src = random_picture(rng, 96, 64, 8)
    r0, r1 = random_picture(rng, 96, 64, 8), random_picture(rng, 96, 64, 8)
    jobs = np.zeros(3, capi.BI_JOB_DTYPE)
    for i, (x, y, w, h, m0, m1) in enumerate([(16, 8, 16, 16, (8, -4), (-12, 4)), (0, 0, 32, 32, (0, 0), (4, 4)),
                                              (48, 16, 32, 32, (-16, 8), (16, -8))]):
        jobs[i]["x"], jobs[i]["y"], jobs[i]["w"], jobs[i]["h"] = x, y, w, h
        jobs[i]["ref"] = (0, 1)
        jobs[i]["mv"] = (m0, m1)
    got = oracle.hevc_bi(8, src, [r0, r1], oracle.params(HEVC, 32), jobs, refine=False)
    for j, g in zip(jobs, got):
        x, y, w, h = (int(j[k]) for k in ("x", "y", "w", "h"))
        (ax, ay), (bx, by) = (j["mv"][0] // 4), (j["mv"][1] // 4)
        a = r0[y + ay:y + ay + h, x + ax:x + ax + w].astype(np.int64)
        b = r1[y + by:y + by + h, x + bx:x + bx + w].astype(np.int64)
        assert g == _satd(src[y:y + h, x:x + w], (a + b + 1) >> 1)


def test_bi_satd_of_one_vector_twice_is_its_uni_satd():
    """Both forms agree when the pair is one vector twice: the rounded
    average of a block with itself, and bi of two equal 14-bit predictions
    (which rounds as uni does)."""
    rng = np.random.default_rng(2)
    src = random_picture(rng, 128, 96, 10)
    ref = random_picture(rng, 128, 96, 10)
    p = oracle.params(HEVC, 30)
    for mv in [(5, -3), (-2, 7), (400, 9), (-700, -500)]:  # the last two leave HalfPlanes' reach
        jobs = np.zeros(1, capi.BI_JOB_DTYPE)
        jobs[0]["x"], jobs[0]["y"], jobs[0]["w"], jobs[0]["h"] = 32, 16, 16, 16
        jobs[0]["ref"] = (0, 0)
        jobs[0]["mv"] = (mv, mv)
        got = oracle.hevc_bi(10, src, [ref], p, jobs, refine=False)[0]
        pred = oracle.hevc_predict(ref, 10, 32, 16, mv[0], mv[1], 16, 16)
        assert got == _satd(src[16:32, 32:48], pred)


def test_refine_bi_finds_the_list_that_completes_the_target():
    """With list 1 predicting the source exactly (its reference is the source
    itself at the zero vector), the target 2 * src - pred is the source, so
    list 0's search finds the true translation of its reference, at no
    SATD."""
    rng = np.random.default_rng(3)
    ref0 = random_picture(rng, 192, 128, 8)
    src = shifted(ref0, 6, -4)
    jobs = np.zeros(2, capi.BI_JOB_DTYPE)
    for i, (x, y) in enumerate([(64, 48), (96, 32)]):
        jobs[i]["x"], jobs[i]["y"], jobs[i]["w"], jobs[i]["h"] = x, y, 16, 16
        jobs[i]["ref"] = (0, 1)
        jobs[i]["mv"] = ((5 * 4, -3 * 4), (0, 0))  # list 0 starts a sample off
        jobs[i]["list"] = 0
        jobs[i]["mvp"] = ((0, 0), (0, 0))
    got = oracle.hevc_bi(8, src, [ref0, src], oracle.params(HEVC, 32), jobs, refine=True)
    assert (got["mvx"] == 24).all() and (got["mvy"] == -16).all()
    assert (got["satd"] == 0).all() and (got["ref"] == 0).all()


def test_bi_jobs_are_checked():
    rng = np.random.default_rng(4)
    src = random_picture(rng, 64, 64, 8)
    jobs = _jobs(rng, 64, 64, 1)
    jobs[0]["ref"] = (0, 2)
    with pytest.raises(RuntimeError):
        oracle.hevc_bi(8, src, [src, src], oracle.params(HEVC, 32), jobs, refine=False)


def _upload(ms, src, refs, bd, base):
    ms.upload(base, src, HEVC, bd, as_ref=False)
    for i, r in enumerate(refs):
        ms.upload(base + 1 + i, r, HEVC, bd, as_ref=True)
    return [base + 1 + i for i in range(len(refs))]


@pytest.mark.gpu
@pytest.mark.parametrize("bd,w,h", [(8, 352, 288), (10, 416, 240), (8, 1920, 1152)])
def test_bi_kernels_match_the_oracle(ms, bd, w, h):
    """Both kernels over random pairs, some far outside HalfPlanes' reach
    (the exact bi-prediction); 1920x1152 is above HalfPlanes' quarter limit,
    so its quarter phases are never read and those pairs take the exact
    form too."""
    rng = np.random.default_rng(bd * 100 + w)
    r0 = random_picture(rng, w, h, bd)
    r1 = shifted(r0, -7, 5, rng, 1.0)
    src = shifted(r0, 5, -3, rng, 2.0)
    ids = _upload(ms, src, [r0, r1], bd, 1300)
    p = oracle.params(HEVC, 32)
    jobs = _jobs(rng, w, h, 300 if w < 1000 else 120, far=0.15)
    got = ms.bi_satd(1300, ids, p, jobs)
    want = oracle.hevc_bi(bd, src, [r0, r1], p, jobs, refine=False)
    bad = np.nonzero(got != want)[0]
    assert len(bad) == 0, f"{len(bad)} SATDs differ; first {bad[:5]}: {got[bad[:5]]} vs {want[bad[:5]]}"
    got_r = ms.bi_refine(1300, ids, p, jobs)
    want_r = oracle.hevc_bi(bd, src, [r0, r1], p, jobs, refine=True)
    assert_results_equal(got_r, want_r, "refine_bi")
    for i in range(3):
        ms.release(1300 + i)


@pytest.mark.gpu
def test_refine_bi_on_the_device_finds_the_translation(ms):
    rng = np.random.default_rng(3)
    ref0 = random_picture(rng, 192, 128, 8)
    src = shifted(ref0, 6, -4)
    ids = _upload(ms, src, [ref0, src], 8, 1400)
    jobs = np.zeros(2, capi.BI_JOB_DTYPE)
    for i, (x, y) in enumerate([(64, 48), (96, 32)]):
        jobs[i]["x"], jobs[i]["y"], jobs[i]["w"], jobs[i]["h"] = x, y, 16, 16
        jobs[i]["ref"] = (0, 1)
        jobs[i]["mv"] = ((20, -12), (0, 0))
    got = ms.bi_refine(1400, ids, oracle.params(HEVC, 32), jobs)
    assert (got["mvx"] == 24).all() and (got["mvy"] == -16).all() and (got["satd"] == 0).all()
    for i in range(3):
        ms.release(1400 + i)


def test_weighted_bi_with_one_list_is_the_plain_block():
    """Explicit weighting with w1 = 0, w0 = 2^(denom + 1) and log2_wd =
    denom + 14 - bd keeps list 0's 14-bit prediction alone, rounded back to the
    sample depth: at a whole-sample vector the reference block itself, so
    the score is the SATD against that block, whatever list 1 holds."""
    rng = np.random.default_rng(31)
    for bd in (8, 10):
        src, r0, r1 = (random_picture(rng, 96, 64, bd) for _ in range(3))
        jobs = np.zeros(3, capi.BI_JOB_DTYPE)
        for i, (x, y, w, h, m0, m1) in enumerate([(16, 8, 16, 16, (8, -4), (-13, 6)),
                                                  (0, 0, 32, 32, (0, 0), (1203, -7)),
                                                  (48, 16, 32, 32, (-16, 8), (17, -9))]):
            jobs[i]["x"], jobs[i]["y"], jobs[i]["w"], jobs[i]["h"] = x, y, w, h
            jobs[i]["ref"] = (0, 1)
            jobs[i]["mv"] = (m0, m1)
        denom = 5
        got = oracle.hevc_bi_weighted(bd, src, [r0, r1], oracle.params(HEVC, 32), jobs,
                                      (denom + 14 - bd, 2 << denom, 0, 0, 0))
        for j, g in zip(jobs, got):
            x, y, w, h = (int(j[k]) for k in ("x", "y", "w", "h"))
            ax, ay = j["mv"][0] // 4
            assert g == _satd(src[y:y + h, x:x + w], r0[y + ay:y + ay + h, x + ax:x + ax + w])


def test_identity_weighting_is_the_exact_bi_prediction():
    """w0 = w1 = 2^denom, no offsets, log2_wd = denom + 14 - bd is
    (a + b + 2^(14 - bd)) >> (15 - bd), the default bi: equal to the
    default score wherever that score takes the exact form (a vector out
    of HalfPlanes' reach), and an offset pair shifts every sample."""
    rng = np.random.default_rng(32)
    src, r0, r1 = (random_picture(rng, 128, 96, 10) for _ in range(3))
    p = oracle.params(HEVC, 32)
    jobs = _jobs(rng, 128, 96, 60)
    jobs["mv"][:, 1, 0] = rng.integers(800, 1200, size=60) * rng.choice([-1, 1], size=60)
    want = oracle.hevc_bi(10, src, [r0, r1], p, jobs, refine=False)
    for denom in (0, 3, 7):
        got = oracle.hevc_bi_weighted(10, src, [r0, r1], p, jobs, (denom + 4, 1 << denom, 1 << denom, 0, 0))
        np.testing.assert_array_equal(got, want)
    flat = np.full_like(src, 512)
    r = oracle.hevc_bi_weighted(10, flat, [flat, flat], p, jobs[:4], (4, 1, 1, 7, 5))
    # Flat references and source: every sample predicts 512 + 6, the SATD of
    # a constant difference 6 is 16 * 6 / 2 per 4x4 tile (its DC term).
    assert list(r) == [(int(j["w"]) * int(j["h"]) // 16) * 48 for j in jobs[:4]]


def test_weighted_bi_jobs_are_checked():
    rng = np.random.default_rng(33)
    pic = random_picture(rng, 64, 64, 8)
    jobs = _jobs(rng, 64, 64, 2)
    for wt in [(15, 1, 1, 0, 0), (6, 300, 1, 0, 0), (6, 1, -129, 0, 0), (6, 1, 1, 5000, 0)]:
        with pytest.raises(RuntimeError):
            oracle.hevc_bi_weighted(8, pic, [pic, pic], oracle.params(HEVC, 32), jobs, wt)


@pytest.mark.gpu
@pytest.mark.parametrize("bd,w,h,wt", [(8, 352, 288, (7, 90, 40, 3, -9)), (10, 416, 240, (5, -20, 70, 100, 4)),
                                       (8, 1920, 1152, (6, 64, 64, 0, 0))])
def test_weighted_bi_satd_matches_the_oracle(ms, bd, w, h, wt):
    rng = np.random.default_rng(bd * 7 + w)
    r0 = random_picture(rng, w, h, bd)
    r1 = shifted(r0, -7, 5, rng, 1.0)
    src = shifted(r0, 5, -3, rng, 2.0)
    ids = _upload(ms, src, [r0, r1], bd, 1350)
    p = oracle.params(HEVC, 32)
    jobs = _jobs(rng, w, h, 300 if w < 1000 else 120, far=0.15)
    got = ms.bi_satd_weighted(1350, ids, p, jobs, *wt)
    want = oracle.hevc_bi_weighted(bd, src, [r0, r1], p, jobs, wt)
    bad = np.nonzero(got != want)[0]
    assert len(bad) == 0, f"{len(bad)} SATDs differ; first {bad[:5]}: {got[bad[:5]]} vs {want[bad[:5]]}"
    for i in range(3):
        ms.release(1350 + i)
