"""The lookahead's half-resolution ME (HEVC: encode/h265_cutree.rs; H.264:
encode/h264_lookahead.rs): the oracle's restatement against the reference's
properties on the CPU, and the device kernels against the oracle, block for
block."""
import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
from _common import random_picture, shifted

HEVC = capi.RME_CODEC_HEVC
H264 = capi.RME_CODEC_H264


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


def _lcg_picture(w, h):
    """h265_cutree.rs:322-335's picture: s = s * 1103515245 + 12345 (32-bit),
    each sample the top byte of s."""
    s, out = 1, np.empty(w * h, np.uint8)
    for i in range(w * h):
        s = (s * 1103515245 + 12345) & 0xFFFFFFFF
        out[i] = s >> 24
    return out.reshape(h, w)


@pytest.mark.parametrize("codec", [HEVC, H264])
def test_a_picture_matches_itself_at_zero_cost(codec):
    """h265_cutree.rs:322-347: searched against itself, every block costs 0
    at the zero vector (both lookaheads)."""
    y = _lcg_picture(64, 64)
    cost, mv, _ = oracle.lowres_search(y, y, 8, codec=codec)
    assert (cost == 0).all() and (mv == 0).all()


def test_h264_lowres_plane_keeps_the_sample_type():
    """Lookahead::add (h264_lookahead.rs:87-117): 8 samples per macroblock,
    each the rounded 2x2 mean at the stream's depth (no shift), columns and
    rows clamped to the picture, the 24-sample border replicated."""
    rng = np.random.default_rng(4)
    pic = random_picture(rng, 70, 46, 10)
    plane, intra = oracle.lowres(pic, 10, H264)
    bw, bh = 5, 3
    assert plane.dtype == np.uint16
    assert plane.shape == (bh * 8 + 48, bw * 8 + 48) and len(intra) == bw * bh
    p = pic.astype(np.int64)
    for yy in (0, 5, 22, 23):
        for xx in (0, 17, 34, 39):
            x0, x1 = min(2 * xx, 69), min(2 * xx + 1, 69)
            y0, y1 = min(2 * yy, 45), min(2 * yy + 1, 45)
            s = p[y0, x0] + p[y0, x1] + p[y1, x0] + p[y1, x1]
            assert plane[yy + 24, xx + 24] == (s + 2) >> 2
    assert (plane[:24] == plane[24]).all() and (plane[:, :24] == plane[:, 24:25]).all()
    assert (intra >= 12).all()


def test_h264_intra_cost_of_a_flat_picture_is_the_constant():
    """A flat picture predicts exactly from DC (its own mean where there are
    no neighbours): every block costs the constant 12."""
    pic = np.full((64, 96), 77, np.uint8)
    _, intra = oracle.lowres(pic, 8, H264)
    assert (intra == 12).all()


def test_h264_lowres_search_finds_a_translation():
    """A picture moved by (12, -8) samples is found at (6, -4) half-resolution
    samples by the hexagon and square, away from the edges, at no cost."""
    rng = np.random.default_rng(11)
    ref = random_picture(rng, 256, 160, 8)
    cur = np.ascontiguousarray(np.roll(np.roll(ref, -8, axis=0), 12, axis=1))
    cost, mv, nsad = oracle.lowres_search(cur, ref, 8, H264)
    bw = 16
    inner = [by * bw + bx for by in range(2, 8) for bx in range(3, 13)]
    assert (mv[inner] == np.array([-6, 4], np.int16)).all()
    assert (cost[inner] == 0).all()
    # The zero vector, the hexagon's first six points and the square at least.
    assert (nsad >= 1 + 8).all()
    # Vectors stay in the window: 16 samples into the border, 32 at most.
    assert (np.abs(mv) <= 32).all()


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


@pytest.mark.gpu
@pytest.mark.parametrize("bd,w,h", [(8, 1920, 1080), (10, 352, 288), (8, 200, 134), (12, 136, 72)])
def test_h264_lowres_kernels_match_the_oracle(ms, bd, w, h):
    """The H.264 lookahead: plane, intra costs, both lists' searches and the
    average-of-two cost, block for block."""
    rng = np.random.default_rng(bd * 7 + w)
    r0 = random_picture(rng, w, h, bd)
    r1 = shifted(r0, 9, -5, rng, 1.0)
    cur = shifted(r0, -6, 7, rng, 2.0)
    for i, pic in enumerate((cur, r0, r1)):
        ms.upload(900 + i, pic, H264, bd, as_ref=False)
        ms.lowres_build(900 + i)
    _, want_intra = oracle.lowres(cur, bd, H264)
    np.testing.assert_array_equal(ms.lowres_intra(900), want_intra)
    got0 = ms.lowres_search(900, 901)
    want0 = oracle.lowres_search(cur, r0, bd, H264)
    for g, w_, name in zip(got0, want0, ("cost", "mv", "nsad")):
        np.testing.assert_array_equal(g, w_, name)
    got1 = ms.lowres_search(900, 902)
    want1 = oracle.lowres_search(cur, r1, bd, H264)
    for g, w_, name in zip(got1, want1, ("cost", "mv", "nsad")):
        np.testing.assert_array_equal(g, w_, name)
    bi = ms.lowres_bi_cost(900, 901, got0[1], 902, got1[1])
    np.testing.assert_array_equal(bi, oracle.lowres_bi_cost(cur, r0, want0[1], r1, want1[1], bd, H264))
    for i in range(3):
        ms.release(900 + i)


@pytest.mark.gpu
@pytest.mark.parametrize("codec,bd", [(HEVC, 8), (H264, 10)])
def test_lowres_search_batch_equals_pair_by_pair(ms, codec, bd):
    """Many (cur, ref) pairs in one launch: each pair's blocks as its own
    search gives them, and as the oracle's."""
    rng = np.random.default_rng(31 + bd)
    pics = [random_picture(rng, 352, 288, bd)]
    for k in range(4):
        pics.append(shifted(pics[-1], 3 - k, k - 2, rng, 1.5))
    for i, pic in enumerate(pics):
        ms.upload(950 + i, pic, codec, bd, as_ref=False)
        ms.lowres_build(950 + i)
    pairs = [(954, 953), (954, 952), (953, 952), (953, 951), (952, 950), (951, 950)]
    got = ms.lowres_search_batch(pairs)
    for (c, r), g in zip(pairs, got):
        single = ms.lowres_search(c, r)
        for a, b, name in zip(g, single, ("cost", "mv", "nsad")):
            np.testing.assert_array_equal(a, b, name)
    want = oracle.lowres_search(pics[4], pics[3], bd, codec)
    for a, b, name in zip(got[0], want, ("cost", "mv", "nsad")):
        np.testing.assert_array_equal(a, b, name)
    for i in range(len(pics)):
        ms.release(950 + i)


@pytest.mark.gpu
@pytest.mark.parametrize("codec", [HEVC, H264])
def test_a_picture_matches_itself_on_the_device(ms, codec):
    rng = np.random.default_rng(41)
    for k, pic in enumerate((_lcg_picture(64, 64), random_picture(rng, 640, 352, 8))):
        ms.upload(2300 + k, pic, codec, 8, as_ref=False)
        ms.lowres_build(2300 + k)
        cost, mv, nsad = ms.lowres_search(2300 + k, 2300 + k)
        assert (cost == 0).all() and (mv == 0).all()
        want = oracle.lowres_search(pic, pic, 8, codec=codec)
        np.testing.assert_array_equal(nsad, want[2])
        ms.release(2300 + k)
