"""The oracle against the reference's own tests (CPU only).

The reference pins its motion search with property tests, not golden
vectors; they are restated here against the oracle's C++ restatement:
distortion closed forms and the direct Hadamard product
(dsp/distortion.rs:465-576), plane equality against the decoders' direct
interpolation (h264_hpel.rs:1033-1075, h265_search.rs:289-353), and the
translation-found searches (h264_me.rs:3937-4118, h265_me.rs:5222-5369).
The committed golden fixtures freeze the oracle's outputs.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
from _common import lcg_picture, random_picture, shifted

H264, HEVC = capi.RME_CODEC_H264, capi.RME_CODEC_HEVC
GOLDEN = Path(__file__).resolve().parent / "golden"


def lcg_bytes(seed, n):
    """distortion.rs:458-463: s = s*6364136223846793005 + 1442695040888963407, >> 33."""
    out, s = np.zeros(n, np.uint8), seed
    for i in range(n):
        s = (s * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        out[i] = (s >> 33) & 0xFF
    return out


# ---- distortion (dsp/distortion.rs:465-576) -------------------------------------
@pytest.mark.parametrize("simd", [0, 1])
def test_a_block_against_itself_is_zero(simd):
    p = lcg_bytes(5, 64 * 64).reshape(64, 64)
    for w, h in [(4, 4), (8, 8), (16, 16), (16, 8), (8, 16), (64, 64)]:
        assert oracle.sad(8, p[:h, :w], p[:h, :w], simd) == 0
        assert oracle.satd(8, p[:h, :w], p[:h, :w], simd) == 0


@pytest.mark.parametrize("simd", [0, 1])
def test_a_constant_offset_has_a_closed_form(simd):
    for d in (1, 7, 30):
        a = np.full((64, 64), 100, np.uint8)
        b = np.full((64, 64), 100 + d, np.uint8)
        for w, h in [(4, 4), (8, 8), (16, 16), (16, 4)]:
            area = w * h
            assert oracle.sad(8, a[:h, :w], b[:h, :w], simd) == d * area
            assert oracle.satd(8, a[:h, :w], b[:h, :w], simd) == area // 16 * ((16 * d + 1) >> 1)


def test_satd_agrees_with_a_direct_hadamard():
    H = np.array([[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, -1, 1], [1, -1, 1, -1]])
    v = lcg_bytes(99, 200 * 32).reshape(200, 32)
    for k in range(200):
        a = v[k, :16].reshape(4, 4)
        b = v[k, 16:].reshape(4, 4)
        want = int(np.abs(H @ (a.astype(int) - b.astype(int)) @ H.T).sum())
        assert oracle.satd(8, a, b) == (want + 1) >> 1


def test_strides_are_honoured():
    wide = lcg_bytes(21, 64 * 64).reshape(64, 64)
    other = lcg_bytes(22, 64 * 64).reshape(64, 64)
    a, b = wide[3:11, 5:13], other[3:11, 5:13]
    pa, pb = np.ascontiguousarray(a), np.ascontiguousarray(b)
    assert oracle.sad(8, a, b) == oracle.sad(8, pa, pb)
    assert oracle.satd(8, a, b) == oracle.satd(8, pa, pb)


@pytest.mark.parametrize("simd", [0, 1])
def test_wide_samples_do_not_overflow(simd):
    a = np.zeros((64, 64), np.uint16)
    b = np.full((64, 64), 1023, np.uint16)
    assert oracle.sad(10, a, b, simd) == 1023 * 4096
    assert oracle.satd(10, a, b, simd) == 256 * ((16 * 1023 + 1) >> 1)


@pytest.mark.parametrize("bd", [8, 10, 12])
def test_the_avx2_rungs_equal_the_scalar_kernels(bd):
    """The timed CPU baseline uses AVX2 rungs: they must be the scalar
    kernels exactly (as the reference checks every SIMD rung)."""
    rng = np.random.default_rng(bd)
    dt = np.uint8 if bd == 8 else np.uint16
    for _ in range(60):
        w = int(rng.choice([4, 8, 12, 16, 24, 32, 40, 48, 56, 64]))
        h = int(rng.choice([4, 8, 12, 16, 24, 32, 48, 64]))
        a = rng.integers(0, 1 << bd, size=(70, 80)).astype(dt)
        b = rng.integers(0, 1 << bd, size=(70, 80)).astype(dt)
        x, y = int(rng.integers(0, 80 - w)), int(rng.integers(0, 70 - h))
        sa, sb = a[y:y + h, x:x + w], b[y:y + h, x:x + w]
        assert oracle.sad(bd, sa, sb, 1) == oracle.sad(bd, sa, sb, 0)
        assert oracle.satd(bd, sa, sb, 1) == oracle.satd(bd, sa, sb, 0)


@pytest.mark.parametrize("bd", [8, 10, 12])
@pytest.mark.parametrize("w,h,force", [(200, 120, True), (96, 64, False), (131, 77, True)])
def test_the_avx2_interpolation_rung_builds_the_same_planes(bd, w, h, force):
    """The timed CPU baseline builds HalfPlanes with AVX2 qpel_h / qpel_v /
    qpel_v2 / uni passes: every phase plane must be the scalar one exactly,
    tile edges and ragged widths included."""
    rng = np.random.default_rng(100 + bd + w)
    pic = rng.integers(0, 1 << bd, size=(h, w)).astype(np.uint8 if bd == 8 else np.uint16)
    a, ea = oracle.hevc_planes(pic, bd, force_quarter=force, simd=0)
    b, eb = oracle.hevc_planes(pic, bd, force_quarter=force, simd=1)
    assert ea == eb
    np.testing.assert_array_equal(a, b)


# ---- planes -----------------------------------------------------------------------
QPEL = [(0, 0, 0, -1, 0, 0), (0, 0, 0, 1, 0, 0), (1, 0, 0, -1, 0, 0), (1, 0, 0, 0, 1, 0),
        (0, 0, 0, 2, 0, 0), (1, 0, 0, 2, 0, 0), (1, 0, 0, 3, 0, 0), (1, 0, 0, 2, 1, 0),
        (2, 0, 0, -1, 0, 0), (2, 0, 0, 3, 0, 0), (3, 0, 0, -1, 0, 0), (3, 0, 0, 2, 1, 0),
        (2, 0, 0, 0, 0, 1), (2, 0, 0, 1, 0, 1), (3, 0, 0, 1, 0, 1), (2, 1, 0, 1, 0, 1)]


def test_h264_plane_predictions_are_the_decoders():
    """h264_hpel.rs:1033-1075: every quarter-sample vector in [-12, 12)^2 of
    a 16x16 block at (16, 8) of a 48x40 LCG plane, fetched through the half
    planes, equals the decoder's direct 8.4.2.2.1 evaluation."""
    pic = lcg_picture(48, 40, 12345)
    planes = oracle.h264_planes(pic, 8).astype(np.int32)
    pad = 32
    bx, by = 16, 8
    for my in range(-12, 12):
        for mx in range(-12, 12):
            xi, yi = bx + (mx >> 2), by + (my >> 2)
            p1, dx1, dy1, p2, dx2, dy2 = QPEL[(my & 3) * 4 + (mx & 3)]
            a = planes[p1][pad + yi + dy1:pad + yi + dy1 + 16, pad + xi + dx1:pad + xi + dx1 + 16]
            if p2 >= 0:
                b = planes[p2][pad + yi + dy2:pad + yi + dy2 + 16, pad + xi + dx2:pad + xi + dx2 + 16]
                a = (a + b + 1) >> 1
            want = oracle.h264_qpel_direct(pic, 8, xi, yi, mx & 3, my & 3, 16, 16)
            np.testing.assert_array_equal(a, want, err_msg=f"mv ({mx}, {my})")


def test_hevc_half_planes_equal_the_decoders_interpolation():
    """h265_search.rs:289-353: every phase at every position equals
    predict_block's uni-predicted output."""
    pic = lcg_picture(40, 24, 7)
    planes, ext = oracle.hevc_planes(pic, 8, force_quarter=True)
    pad = 80
    for mvx, mvy in [(2, 0), (0, 2), (2, 2), (-6, 10), (14, -2), (-30, -30), (1, 0), (0, 3), (1, 1), (3, 2),
                     (-7, 5), (13, -11)]:
        for x, y in [(0, 0), (8, 4), (32, 16)]:
            xi, yi = x + (mvx >> 2), y + (mvy >> 2)
            if xi < -ext or yi < -ext or xi + 8 > 40 + ext or yi + 8 > 24 + ext:
                continue
            ph = (mvy & 3) * 4 + (mvx & 3)
            got = planes[ph][pad + yi:pad + yi + 8, pad + xi:pad + xi + 8]
            want = oracle.hevc_predict(pic, 8, x, y, mvx, mvy, 8, 8)
            np.testing.assert_array_equal(got, want, err_msg=f"mv ({mvx},{mvy}) at ({x},{y})")


def test_hevc_quarter_phases_are_dropped_above_the_limit():
    """h265_search.rs:33-35: above 2.2 Msamples only the 3 half phases."""
    pic = np.zeros((1090, 2048), np.uint8)
    planes, _ = oracle.hevc_planes(pic + 1, 8)
    built = [k for k in range(1, 16) if planes[k].any()]
    assert built == [2, 8, 10]


# ---- rate model ---------------------------------------------------------------------
def test_the_mv_bits_closed_form_equals_the_model():
    """The device's mvd bits, 1 at zero else 3 + 2 floor(log2 |d|), equal
    mvd_bits_of's Exp-Golomb loop (h265_search.rs:232-247) for every |d|."""
    import ctypes as C
    pq = (C.c_int32 * 4)(0, 0, 0, 0)
    for d in list(range(0, 5000)) + list(range(5000, 65536, 37)):
        loop = oracle.lib().orc_hevc_mv_bits(d, 0, pq) - 2  # one component (the other is 0: 1 bit), + 1 flag
        closed = 1 if d == 0 else 3 + 2 * (d.bit_length() - 1)
        assert loop == closed, d


def test_the_h264_rate_table_is_symmetric_and_monotone():
    import ctypes as C
    tab = (C.c_uint16 * 8193)()
    oracle.lib().orc_h264_cost_table(oracle.lib().orc_h264_lambda(28), tab)
    t = np.array(tab)
    assert (t[4096:] == t[4096::-1]).all()
    assert (np.diff(t[4096:]) >= 0).all()


# ---- search behaviour -------------------------------------------------------------------
def grating(w, h):
    y, x = np.mgrid[0:h, 0:w]
    return (40 + 4 * np.abs(x % 25 - 12) + 3 * np.abs(y % 27 - 13)).astype(np.uint8)


def test_hevc_an_integral_translation_is_found_exactly():
    """h265_me.rs:5222-5262: the grating moved by (-6, 4), 32x32 units."""
    ref = grating(64, 32)
    src = shifted(ref, -6, 4)
    res = oracle.frame_search(HEVC, 8, src, [ref], oracle.params(HEVC, 26, hevc_pu_mask=0b0100))
    assert (res["mvx"] == -24).all() and (res["mvy"] == 16).all()


def test_hevc_a_half_sample_translation_is_found_by_the_refinement():
    """h265_me.rs:5301-5350: the decoder's own (2, 0) interpolation."""
    ref = grating(64, 32)
    src = oracle.hevc_predict(ref, 8, 0, 0, 2, 0, 64, 32)
    res = oracle.frame_search(HEVC, 8, src, [ref], oracle.params(HEVC, 26, hevc_pu_mask=0b0010))
    assert (res["mvx"] == 2).all() and (res["mvy"] == 0).all() and (res["satd"] == 0).all()


@pytest.mark.parametrize("d", [(0, 0), (1, 0), (0, -1), (5, 3), (-7, 2), (3, -8), (8, 8), (-8, -8)])
def test_h264_an_integral_translation_is_found_exactly(d):
    """h264_me.rs:3937-3990: a 3x3-macroblock grating picture; the centre
    macroblock finds the translation (zero-seeded walks stay at |d| <= 8,
    inside the true basin)."""
    ref = grating(48, 48)
    res = oracle.frame_search(H264, 8, shifted(ref, *d), [ref], oracle.params(H264, 26))
    assert (res[4]["mvx"], res[4]["mvy"]) == (d[0] * 4, d[1] * 4)


def test_h264_the_search_keeps_the_levels_vertical_range():
    """h264_me.rs:3802: with vertical_search v every vector's vertical
    component stays within +-v whole samples."""
    rng = np.random.default_rng(3)
    ref = random_picture(rng, 96, 96, 8)
    src = shifted(ref, 2, 14, rng, 1.0)
    for v in (0, 3, 8):
        res = oracle.frame_search(H264, 8, src, [ref], oracle.params(H264, 26, h264_vertical_range=v))
        assert (np.abs(res["mvy"]) <= 4 * v).all()


# ---- golden fixtures ----------------------------------------------------------------------
@pytest.mark.parametrize("name", ["h264_96x64_medium", "h264_96x64_umh", "hevc_128x96_medium",
                                  "hevc_128x96_rings_cross", "hevc_96x64_10bit"])
def test_the_oracle_reproduces_its_golden_fixtures(name):
    z = np.load(GOLDEN / f"{name}.npz")
    codec, bd = int(z["codec"]), int(z["bit_depth"])
    kw = dict(eval(str(z["params"])))
    p = oracle.params(codec, int(z["qp"]), **kw)
    got = oracle.frame_search(codec, bd, z["src"], list(z["refs"]), p)
    np.testing.assert_array_equal(got.view(np.uint8), z["results"])


def test_the_oracle_reproduces_its_golden_planes():
    z = np.load(GOLDEN / "hevc_planes_96x64_10bit.npz")
    planes, ext = oracle.hevc_planes(z["pic"], 10, force_quarter=True)
    assert ext == int(z["ext"])
    np.testing.assert_array_equal(planes, z["planes"])


def test_simd_and_scalar_searches_agree():
    rng = np.random.default_rng(8)
    ref = random_picture(rng, 128, 96, 8)
    src = shifted(ref, 4, -3, rng, 2.0)
    p = oracle.params(HEVC, 30)
    a = oracle.frame_search(HEVC, 8, src, [ref], p, simd=0)
    b = oracle.frame_search(HEVC, 8, src, [ref], p, simd=1)
    np.testing.assert_array_equal(a, b)
