"""H.264 B macroblocks: b_mb's joint refinement of a vector pair
(encode/h264_analyse.rs:2793-2900). The oracle's restatement against closed
forms on the CPU; the device kernel against the oracle, pair for pair."""
import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
from _common import random_picture, shifted

H264 = capi.RME_CODEC_H264


def _satd(a, b):
    h4 = np.array([[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, -1, 1], [1, -1, 1, -1]])
    d = a.astype(np.int64) - b.astype(np.int64)
    return sum((int(np.abs(h4 @ d[y:y + 4, x:x + 4] @ h4.T).sum()) + 1) >> 1
               for y in range(0, d.shape[0], 4) for x in range(0, d.shape[1], 4))


def _jobs(rng, w, h, n, spread=40, nref=2):
    jobs = np.zeros(n, capi.H264_BI_JOB_DTYPE)
    for i in range(n):
        bw, bh = [(16, 16), (8, 8), (16, 8), (8, 16), (4, 4), (8, 4)][rng.integers(6)]
        jobs[i]["x"] = rng.integers(0, (w - bw) // 4 + 1) * 4
        jobs[i]["y"] = rng.integers(0, (h - bh) // 4 + 1) * 4
        jobs[i]["w"], jobs[i]["h"] = bw, bh
        jobs[i]["ref"] = rng.integers(nref, size=2)
        jobs[i]["mv"] = rng.integers(-spread, spread + 1, size=(2, 2))
        jobs[i]["mvp"] = rng.integers(-spread, spread + 1, size=(2, 2))
        jobs[i]["limit"] = 0xFFFFFFFF if rng.random() < 0.8 else rng.integers(0, 4000)
    return jobs


def _params(qp=30):
    return oracle.params(H264, qp, predictor_mode=capi.RME_PRED_GIVEN)


def test_no_rounds_is_the_start_pairs_cost():
    """Whole-sample start vectors, no rounds: the SATD of the rounded average
    of the two displaced blocks, plus a rate that depends only on the
    vectors and predictors (equal for two blocks with the same ones)."""
    rng = np.random.default_rng(1)
    src, r0, r1 = (random_picture(rng, 96, 64, 8) for _ in range(3))
    jobs = np.zeros(2, capi.H264_BI_JOB_DTYPE)
    for i, (x, y) in enumerate([(32, 16), (64, 32)]):
        jobs[i]["x"], jobs[i]["y"], jobs[i]["w"], jobs[i]["h"] = x, y, 16, 16
        jobs[i]["ref"] = (0, 1)
        jobs[i]["mv"] = ((8, -4), (-12, 4))
        jobs[i]["mvp"] = ((0, 4), (4, 0))
        jobs[i]["limit"] = 0xFFFFFFFF
    mv, cost = oracle.h264_bi_refine(8, src, [r0, r1], _params(), jobs, rounds=0)
    assert (mv == jobs["mv"]).all()
    rates = []
    for (x, y), c in zip([(32, 16), (64, 32)], cost):
        a = r0[y - 1:y + 15, x + 2:x + 18].astype(np.int64)
        b = r1[y + 1:y + 17, x - 3:x + 13].astype(np.int64)
        rates.append(int(c) - _satd(src[y:y + 16, x:x + 16], (a + b + 1) >> 1))
    assert rates[0] == rates[1] > 0


def test_rounds_never_raise_the_cost_and_the_limit_holds():
    rng = np.random.default_rng(2)
    ref = random_picture(rng, 128, 96, 8)
    src = shifted(ref, 2, -1, rng, 1.0)
    p = _params()
    jobs = _jobs(rng, 128, 96, 40, nref=1)
    jobs["limit"] = 0xFFFFFFFF
    _, c0 = oracle.h264_bi_refine(8, src, [ref], p, jobs, rounds=0)
    m2, c2 = oracle.h264_bi_refine(8, src, [ref], p, jobs, rounds=2)
    assert (c2 <= c0).all() and (c2 < c0).any()
    # Each round moves a list's vector a quarter sample at most.
    assert (np.abs(m2.astype(int) - jobs["mv"].astype(int)) <= 2).all()
    jobs["limit"] = 0
    m, c = oracle.h264_bi_refine(8, src, [ref], p, jobs, rounds=2)
    assert (m == jobs["mv"]).all() and (c == c0).all()


def test_a_reachable_vector_outside_the_planes_is_refused():
    rng = np.random.default_rng(3)
    pic = random_picture(rng, 64, 64, 8)
    jobs = _jobs(rng, 64, 64, 1, nref=1)
    jobs[0]["x"], jobs[0]["y"], jobs[0]["w"], jobs[0]["h"] = 0, 0, 16, 16
    jobs[0]["mv"][0] = (-4 * 28, 0)  # search_bounds' lo_x is 4 - 32 = -28
    with pytest.raises(RuntimeError):
        oracle.h264_bi_refine(8, pic, [pic], _params(), jobs, rounds=1)


@pytest.mark.gpu
@pytest.mark.parametrize("bd,w,h,rounds,diamond", [(8, 352, 288, 2, False), (10, 176, 144, 1, True),
                                                    (8, 200, 136, 3, False)])
def test_h264_bi_refine_matches_the_oracle(ms, bd, w, h, rounds, diamond):
    rng = np.random.default_rng(bd * 1000 + w + rounds)
    r0 = random_picture(rng, w, h, bd)
    r1 = shifted(r0, -5, 3, rng, 1.0)
    src = shifted(r0, 3, -2, rng, 2.0)
    ms.upload(1800, src, H264, bd, as_ref=False)
    ms.upload(1801, r0, H264, bd, as_ref=True)
    ms.upload(1802, r1, H264, bd, as_ref=True)
    p = _params(28)
    cw, ch = -(-w // 16) * 16, -(-h // 16) * 16
    jobs = _jobs(rng, cw, ch, 400)
    got_mv, got_c = ms.h264_bi_refine(1800, [1801, 1802], p, jobs, rounds, diamond)
    want_mv, want_c = oracle.h264_bi_refine(bd, src, [r0, r1], p, jobs, rounds, diamond)
    np.testing.assert_array_equal(got_mv, want_mv)
    np.testing.assert_array_equal(got_c, want_c)
    for i in range(3):
        ms.release(1800 + i)
