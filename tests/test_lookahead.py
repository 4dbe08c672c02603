"""The lookahead's half-resolution ME (encode/h265_cutree.rs): the oracle's
restatement against the reference's properties on the CPU, and the device
kernels against the oracle, block for block."""
import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
from _common import random_picture, shifted

HEVC = capi.RME_CODEC_HEVC


def test_lowres_plane_is_the_mean_of_two_by_two_squares():
    """LowRes::new: each sample the rounded mean of a 2x2 square at 8 bits,
    whole 8x8 blocks, the 24-sample border replicated."""
    rng = np.random.default_rng(3)
    pic = random_picture(rng, 70, 46, 10)
    plane, intra = oracle.lowres(pic, 10)
    lw, lh = 35, 23
    bw, bh = 5, 3
    assert plane.shape == (bh * 8 + 48, bw * 8 + 48) and len(intra) == bw * bh
    p = pic.astype(np.int64)
    for yy in (0, 5, 22, 23):
        for xx in (0, 17, 34, 39):
            x2, y2 = 2 * min(xx, lw - 1), 2 * min(yy, lh - 1)
            at = lambda x, y: p[min(y, 45), min(x, 69)]
            s = at(x2, y2) + at(x2 + 1, y2) + at(x2, y2 + 1) + at(x2 + 1, y2 + 1)
            assert plane[yy + 24, xx + 24] == min(((s + 2) >> 2) >> 2, 255)
    assert (plane[:24] == plane[24]).all() and (plane[:, :24] == plane[:, 24:25]).all()
    assert (intra >= 16).all()


def test_lowres_search_finds_a_translation():
    """A picture moved by (12, -8) samples is found at (6, -4) half-resolution
    samples away from the edges, at the least cost."""
    rng = np.random.default_rng(11)
    ref = random_picture(rng, 256, 160, 8)
    cur = np.ascontiguousarray(np.roll(np.roll(ref, -8, axis=0), 12, axis=1))
    cost, mv, nsad = oracle.lowres_search(cur, ref, 8)
    bw = 16
    inner = [by * bw + bx for by in range(2, 8) for bx in range(3, 13)]
    assert (mv[inner] == np.array([-6, 4], np.int16)).all()
    assert (cost[inner] == 0).all()
    assert (nsad > 0).all()




@pytest.mark.gpu
@pytest.mark.parametrize("bd,w,h", [(8, 1920, 1080), (10, 352, 288), (8, 200, 134)])
def test_lowres_kernels_match_the_oracle(ms, bd, w, h):
    rng = np.random.default_rng(bd + w)
    r0 = random_picture(rng, w, h, bd)
    r1 = shifted(r0, 9, -5, rng, 1.0)
    cur = shifted(r0, -6, 7, rng, 2.0)
    for i, pic in enumerate((cur, r0, r1)):
        ms.upload(800 + i, pic, HEVC, bd, as_ref=False)
        ms.lowres_build(800 + i)
    _, want_intra = oracle.lowres(cur, bd)
    np.testing.assert_array_equal(ms.lowres_intra(800), want_intra)
    got0 = ms.lowres_search(800, 801)
    want0 = oracle.lowres_search(cur, r0, bd)
    for g, w_, name in zip(got0, want0, ("cost", "mv", "nsad")):
        np.testing.assert_array_equal(g, w_, name)
    got1 = ms.lowres_search(800, 802)
    want1 = oracle.lowres_search(cur, r1, bd)
    np.testing.assert_array_equal(got1[1], want1[1])
    bi = ms.lowres_bi_cost(800, 801, got0[1], 802, got1[1])
    np.testing.assert_array_equal(bi, oracle.lowres_bi_cost(cur, r0, want0[1], r1, want1[1], bd))
    for i in range(3):
        ms.release(800 + i)
