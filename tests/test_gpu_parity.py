"""CUDA path against the oracle, bit for bit, through the C ABI.

Every comparison is exact: the search is integer arithmetic end to end, so
every vector, reference index, cost, SATD, whole-sample winner and
candidate count must equal the oracle's on the same input.
"""
import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
import rivet_h26x_codecs_b200.synth as synth
from _common import assert_results_equal, lcg_picture, random_jobs, random_picture, shifted

H264, HEVC = capi.RME_CODEC_H264, capi.RME_CODEC_HEVC
pytestmark = pytest.mark.gpu


def _run(ms, codec, bd, src, refs, p, jobs=None, base=1000):
    ms.upload(base, src, codec, bd, as_ref=False)
    ids = []
    for i, r in enumerate(refs):
        ms.upload(base + 1 + i, r, codec, bd, as_ref=True)
        ids.append(base + 1 + i)
    got = ms.search(base, ids, p, jobs)
    want = oracle.frame_search(codec, bd, src, refs, p, jobs)
    return got, want


# ---- planes -----------------------------------------------------------------
@pytest.mark.parametrize("bd", [8, 10])
def test_h264_half_planes_equal_the_oracles(ms, bd):
    pic = lcg_picture(48, 40, 12345, bd)  # the reference test's plane (h264_hpel.rs:1033-1045)
    ms.upload(1, pic, H264, bd, as_ref=True)
    want = oracle.h264_planes(pic, bd)
    rows, cols = want.shape[1:]
    for k in range(4):
        got = ms.plane(1, k)
        assert got.shape == (rows, cols)
        # b and j are computed where the six-tap window fits across; h and j
        # where it fits down (hpel_planes' loops); elsewhere the reference
        # copies G and the search never reads it.
        ys = slice(2, rows - 3) if k in (2, 3) else slice(0, rows)
        xs = slice(2, cols - 3) if k in (1, 3) else slice(0, cols)
        np.testing.assert_array_equal(got[ys, xs], want[k][ys, xs], err_msg=f"plane {k}")


@pytest.mark.parametrize("bd,w,h", [(8, 40, 24), (10, 72, 40), (8, 200, 136)])
def test_hevc_phases_equal_the_oracles(ms, bd, w, h):
    pic = lcg_picture(w, h, 7, bd) if w == 40 else random_picture(np.random.default_rng(w), w, h, bd)
    ms.upload(2, pic, HEVC, bd, as_ref=True)
    want, ext = oracle.hevc_planes(pic, bd, force_quarter=True)
    pad = 80
    sl = (slice(pad - ext, pad + h + ext), slice(pad - ext, pad + w + ext))
    for k in range(16):
        np.testing.assert_array_equal(ms.plane(2, k)[sl], want[k][sl], err_msg=f"phase {k}")


# ---- H.264 ------------------------------------------------------------------
def test_h264_cif_frame_matches_the_oracle(ms):
    """The CIF P-frame workload: 396 macroblocks, medium MeCfg, QP 28."""
    seq = synth.config0()
    p = oracle.params(H264, 28)
    got, want = _run(ms, H264, 8, seq.frames[1], [seq.frames[0]], p)
    assert_results_equal(got, want, "H.264 CIF")


@pytest.mark.parametrize("variant", ["medium", "umh", "dia", "qpel_diamond", "vr", "slow"])
@pytest.mark.parametrize("bd", [8, 10])
def test_h264_settings_match_the_oracle(ms, variant, bd):
    rng = np.random.default_rng(hash((variant, bd)) & 0xFFFF)
    ref0 = random_picture(rng, 160, 112, bd)
    ref1 = shifted(ref0, 3, -2, rng, 2.0)
    ref2 = shifted(ref0, -5, 4, rng, 2.0)
    src = shifted(ref0, 6, 5, rng, 2.0)
    kw = {"medium": {}, "umh": {"h264_umh": 1}, "dia": {"h264_dia": 1, "h264_hpel_iters": 1, "h264_qpel_iters": 1},
          "qpel_diamond": {"h264_qpel_diamond": 1}, "vr": {"h264_vertical_range": 7},
          "slow": {"h264_range": 24}}[variant]
    p = oracle.params(H264, 30, **kw)
    got, want = _run(ms, H264, bd, src, [ref0, ref1, ref2], p)
    assert_results_equal(got, want, f"H.264 {variant} {bd}-bit")


def test_h264_ragged_picture_size(ms):
    """A picture that is not whole macroblocks (coded size rounded up)."""
    rng = np.random.default_rng(5)
    ref = random_picture(rng, 100, 70, 8)
    src = shifted(ref, -3, 2, rng, 1.0)
    got, want = _run(ms, H264, 8, src, [ref], oracle.params(H264, 26))
    assert_results_equal(got, want, "H.264 100x70")


@pytest.mark.parametrize("bd", [8, 10])
def test_h264_given_jobs_match_the_oracle(ms, bd):
    rng = np.random.default_rng(17 + bd)
    ref0 = random_picture(rng, 128, 96, bd)
    ref1 = shifted(ref0, 2, 1, rng, 1.0)
    src = shifted(ref0, -4, 3, rng, 1.0)
    p = oracle.params(H264, 27, predictor_mode=capi.RME_PRED_GIVEN)
    jobs = random_jobs(rng, H264, 128, 96, 2, 300, sizes=((16, 16), (16, 8), (8, 16), (8, 8), (8, 4), (4, 8),
                                                          (4, 4)))
    got, want = _run(ms, H264, bd, src, [ref0, ref1], p, jobs)
    assert_results_equal(got, want, f"H.264 GIVEN {bd}-bit")


# ---- HEVC -------------------------------------------------------------------
@pytest.mark.parametrize("variant", ["medium", "range64_rings", "cross", "levels", "amp", "amp_all_levels"])
@pytest.mark.parametrize("bd", [8, 10])
def test_hevc_frames_match_the_oracle(ms, variant, bd):
    """STANDALONE frames under the search settings, size levels and AMP
    units (2NxnU + nLx2N as the 2160p workload asks, or all four modes over
    a subset of levels), against the oracle."""
    seq = synth.make_sequence(HEVC, 256, 192, bd, 3, 100 + bd, 64, 64, 2.0 if bd == 8 else 6.0)
    kw = {"medium": {}, "range64_rings": {"hevc_search_range": 64, "hevc_search_rings": 1},
          "cross": {"hevc_quarter_cross": 1, "hevc_search_rings": 2}, "levels": {"hevc_pu_mask": 0b1010},
          "amp": {"hevc_amp": 0b0101}, "amp_all_levels": {"hevc_amp": 0xF, "hevc_pu_mask": 0b0111}}[variant]
    p = oracle.params(HEVC, 32, **kw)
    got, want = _run(ms, HEVC, bd, seq.frames[2], [seq.frames[1], seq.frames[0]], p)
    assert_results_equal(got, want, f"HEVC {variant} {bd}-bit")


@pytest.mark.parametrize("bd", [8, 10])
def test_hevc_given_jobs_match_the_oracle(ms, bd):
    rng = np.random.default_rng(99 + bd)
    ref0 = random_picture(rng, 192, 128, bd)
    ref1 = shifted(ref0, -7, 2, rng, 1.0)
    src = shifted(ref0, 5, -6, rng, 1.0)
    p = oracle.params(HEVC, 30, predictor_mode=capi.RME_PRED_GIVEN, hevc_search_rings=1)
    jobs = random_jobs(rng, HEVC, 192, 128, 2, 400, spread=400)
    got, want = _run(ms, HEVC, bd, src, [ref0, ref1], p, jobs)
    assert_results_equal(got, want, f"HEVC GIVEN {bd}-bit")


def test_hevc_1080p_frame_matches_the_oracle(ms):
    """One frame of the 1080p workload at full size: 42,900 PUs x 2 refs."""
    seq = synth.config1(nframes=3)
    p = oracle.params(HEVC, 32, hevc_search_range=64)
    got, want = _run(ms, HEVC, 8, seq.frames[2], [seq.frames[1], seq.frames[0]], p)
    assert_results_equal(got, want, "HEVC 1080p")
    st = ms.stats()
    assert st.tasks == len(got)
    assert st.sad_candidates == int(want["n_sad"].sum())
    assert st.satd_candidates == int(want["n_satd"].sum())


def test_hevc_4k_10bit_four_references_match_the_oracle(ms):
    """One frame of the 2160p 10-bit workload: four references, +-128,
    10-bit samples, 2Nx2N PUs 8..64 plus the 2NxnU and nLx2N units."""
    seq = synth.config2(nframes=5)
    p = oracle.params(HEVC, 32, hevc_search_range=128, hevc_amp=0b0101)
    f = seq.frames
    got, want = _run(ms, HEVC, 10, f[4], [f[3], f[2], f[1], f[0]], p, base=2000)
    assert_results_equal(got, want, "HEVC 2160p 10-bit 4 refs")
    for i in range(2000, 2005):
        ms.release(i)


def test_mixed_stream_batch_equals_the_per_frame_path(ms):
    """The batched form's mix (config 3): H.264 360p 8-bit, HEVC 720p 8-bit,
    HEVC 1080p 10-bit and HEVC 2160p 8-bit streams, two references each and
    ranges 32 / 64 / 64 / 128, one frame of each in one launch (two kinds of
    8-bit task and one 16-bit kind, concurrent); every frame equals its
    per-frame search, and the two smaller ones the oracle."""
    kinds = [(H264, 8, 640, 360, 32), (HEVC, 8, 1280, 720, 64), (HEVC, 10, 1920, 1080, 64), (HEVC, 8, 3840, 2160, 128)]
    frames, params, pics = [], [], {}
    for k, (codec, bd, w, h, rng_) in enumerate(kinds):
        seq = synth.stream_sequence(codec, w, h, bd, 3, k)
        base = 3000 + 10 * k
        for t, fr in enumerate(seq.frames):
            ms.upload(base + t, fr, codec, bd, as_ref=True)
        pics[k] = seq.frames
        frames.append((base + 2, [base + 1, base]))
        p = oracle.params(codec, 30)
        if codec == HEVC:
            p.hevc_search_range = rng_
        else:
            p.h264_range = rng_
        params.append(p)
    for _ in range(2):
        outs = ms.search_batch(frames, params)
        for (s_id, refs), pp, got in zip(frames, params, outs):
            assert_results_equal(got, ms.search(s_id, refs, pp), f"mix vs per-frame {s_id}")
    for k in (0, 1):
        codec, bd = kinds[k][0], kinds[k][1]
        want = oracle.frame_search(codec, bd, pics[k][2], [pics[k][1], pics[k][0]], params[k])
        assert_results_equal(outs[k], want, f"mix vs oracle {k}")
    for k in range(4):
        for t in range(3):
            ms.release(3000 + 10 * k + t)


def test_throughput_launch_shapes_equal_the_per_frame_path():
    """Four 1080p HEVC frames in one launch (343,200 tasks: the throughput
    form), on every launch shape the tuner times (three occupancies, each
    twice), then on the chosen one: every frame equals its per-frame search
    (the latency form's row form) every time."""
    import rivet_h26x_codecs_b200 as rme
    seq = synth.make_sequence(HEVC, 1920, 1080, 8, 6, 91, 64, 160, 2.0)
    p = oracle.params(HEVC, 32, hevc_search_range=64)
    with rme.MotionSearch(0) as ms2:
        for i, f in enumerate(seq.frames):
            ms2.upload(i, f, HEVC, 8, as_ref=True)
        frames = [(t, [t - 1, t - 2]) for t in range(2, 6)]
        want = [ms2.search(t, refs, p) for t, refs in frames]
        for k in range(2 * 3 + 1):
            outs = ms2.search_batch(frames, p)
            for j, (g, w) in enumerate(zip(outs, want)):
                assert_results_equal(g, w, f"launch {k} frame {j}")


def test_batch_equals_the_frames_and_the_oracle(ms):
    """Several frames of two formats in one persistent launch, three times
    (the second launch captures a graph, the third replays it)."""
    seq = synth.make_sequence(HEVC, 192, 128, 8, 5, 31, 64, 64, 2.0)
    h264 = synth.make_sequence(H264, 96, 64, 8, 3, 32, 16, 32, 2.0)
    ph = oracle.params(HEVC, 32, hevc_search_range=40)
    p4 = oracle.params(H264, 28)
    for i, f in enumerate(seq.frames):
        ms.upload(300 + i, f, HEVC, 8, as_ref=True)
    for i, f in enumerate(h264.frames):
        ms.upload(400 + i, f, H264, 8, as_ref=True)
    frames = [(300 + t, [300 + t - 1, 300 + t - 2]) for t in range(2, 5)] + [(402, [401, 400])]
    params = [ph, ph, ph, p4]
    for _ in range(3):
        outs = ms.search_batch(frames, params)
        for (s, refs), pp, got in zip(frames, params, outs):
            single = ms.search(s, refs, pp)
            assert_results_equal(got, single, f"batch vs single {s}")
            seqf = seq.frames if s < 400 else h264.frames
            base = 300 if s < 400 else 400
            codec = HEVC if s < 400 else H264
            want = oracle.frame_search(codec, 8, seqf[s - base], [seqf[r - base] for r in refs], pp)
            assert_results_equal(got, want, f"batch vs oracle {s}")


def test_batch_results_into_device_and_pinned_memory(ms):
    """The batched search writing its results to a device tensor (they stay
    there) and to pinned host memory (one direct copy) equals the host-array
    form."""
    import torch
    seq = synth.make_sequence(HEVC, 192, 128, 8, 4, 33, 64, 64, 2.0)
    p = oracle.params(HEVC, 30)
    for i, f in enumerate(seq.frames):
        ms.upload(500 + i, f, HEVC, 8, as_ref=True)
    frames = [(500 + t, [500 + t - 1]) for t in range(1, 4)]
    want = ms.search_batch(frames, p)
    n = ms.batch_result_count(frames, p)
    dev = torch.zeros(n * 32 + 64, dtype=torch.uint8, device="cuda:0")
    pin = torch.zeros(n * 32, dtype=torch.uint8, pin_memory=True)
    for _ in range(2):
        got_dev = ms.search_batch(frames, p, out=dev)
        got_pin = ms.search_batch(frames, p, out=pin)
        for w, d, q in zip(want, got_dev, got_pin):
            assert_results_equal(d.cpu().numpy().view(capi.RESULT_DTYPE), w, "device out")
            assert_results_equal(q.numpy().view(capi.RESULT_DTYPE), w, "pinned out")
    with pytest.raises(ValueError):
        ms.search_batch(frames, p, out=torch.zeros(n * 32 - 1, dtype=torch.uint8, device="cuda:0"))


# ---- chroma of chosen vectors and the batched distortion kernels ------------------
@pytest.mark.parametrize("codec,bd", [(HEVC, 8), (HEVC, 10), (H264, 8), (H264, 10)])
def test_chroma_prediction_matches_the_oracle(ms, codec, bd):
    """4:2:0 chroma of chosen luma vectors: HEVC's 4-tap eighth-sample
    filter with uni rounding, H.264's bilinear weights; vectors reaching far
    outside the picture read the edge-replicated planes."""
    import torch
    rng = np.random.default_rng(70 + 2 * bd + codec)
    W, H = 96, 64
    luma = random_picture(rng, W, H, bd)
    cb, cr = random_picture(rng, W // 2, H // 2, bd), random_picture(rng, W // 2, H // 2, bd)
    ms.upload(700, luma, codec, bd, as_ref=True)
    ms.upload_chroma(700, cb, cr)
    sizes = [(8, 8), (16, 16), (32, 32), (64, 64), (16, 8), (8, 16), (4, 4), (2, 2), (12, 6)]
    blocks, mvs = [], []
    for i in range(300):
        bw, bh = sizes[i % len(sizes)]
        blocks.append((rng.integers(0, W - bw + 1), rng.integers(0, H - bh + 1), bw, bh))
        spread = 40 if i % 3 else 600
        mvs.append(rng.integers(-spread, spread + 1, size=2))
    blocks, mvs = np.array(blocks, np.int32), np.array(mvs, np.int16)
    want = oracle.chroma_predict(codec, bd, W, H, cb, cr, blocks, mvs)
    got = ms.chroma_predict(700, blocks, mvs)
    np.testing.assert_array_equal(got, want)
    ms.release(700)


@pytest.mark.parametrize("bd", [8, 10])
@pytest.mark.parametrize("kind", ["sad", "satd"])
def test_distortion_batches_match_the_oracle(kind, bd):
    """rme_sad_batch / rme_satd_batch over device buffers equal the
    reference's size-generic kernels block for block."""
    import torch
    import rivet_h26x_codecs_b200.host as host
    rng = np.random.default_rng(90 + bd + (kind == "satd"))
    A, B = random_picture(rng, 160, 120, bd), random_picture(rng, 160, 120, bd)
    view = np.uint8 if bd == 8 else np.int16
    da = torch.from_numpy(A.view(view).copy()).cuda()
    db = torch.from_numpy(B.view(view).copy()).cuda()
    shapes = [(4, 4), (8, 8), (16, 16), (64, 64), (8, 4), (16, 12), (32, 64)] + ([(3, 5), (7, 1)] if kind == "sad" else [])
    for w, h in shapes:
        n = 97
        ax, ay = rng.integers(0, 160 - w + 1, n), rng.integers(0, 120 - h + 1, n)
        bx, by = rng.integers(0, 160 - w + 1, n), rng.integers(0, 120 - h + 1, n)
        aoff = torch.from_numpy((ay * 160 + ax).astype(np.int64)).cuda()
        boff = torch.from_numpy((by * 160 + bx).astype(np.int64)).cuda()
        out = torch.zeros(n, dtype=torch.int32, device="cuda")
        host.distortion_batch(kind, da, 160, aoff, db, 160, boff, w, h, bd, out)
        got = out.cpu().numpy().view(np.uint32)
        fn = oracle.sad if kind == "sad" else oracle.satd
        want = [fn(bd, A[ay[i]:ay[i] + h, ax[i]:ax[i] + w], B[by[i]:by[i] + h, bx[i]:bx[i] + w]) for i in range(n)]
        np.testing.assert_array_equal(got, np.array(want, np.uint32), f"{kind} {w}x{h}")


# ---- the reference's search-behaviour tests, through the library --------------
def grating(w, h):
    """The reference tests' triangle grating (h265_me.rs:4989-5026,
    h264_me.rs:3698-3710): 40 + 4|x%25-12| + 3|y%27-13|."""
    y, x = np.mgrid[0:h, 0:w]
    return (40 + 4 * np.abs(x % 25 - 12) + 3 * np.abs(y % 27 - 13)).astype(np.uint8)


def test_hevc_integral_translation_is_found_exactly(ms):
    ref = grating(64, 32)
    src = shifted(ref, -6, 4)
    p = oracle.params(HEVC, 26, hevc_pu_mask=0b0100)  # 32x32 units, as the reference test's CTBs
    got, want = _run(ms, HEVC, 8, src, [ref], p)
    assert_results_equal(got, want, "translation")
    assert (got["mvx"] == -24).all() and (got["mvy"] == 16).all(), got[["mvx", "mvy"]]


def test_hevc_half_sample_translation_is_found_by_the_refinement(ms):
    ref = grating(64, 32)
    src = oracle.hevc_predict(ref, 8, 0, 0, 2, 0, 64, 32)  # the decoder's own (2, 0) interpolation
    p = oracle.params(HEVC, 26, hevc_pu_mask=0b0010)
    got, want = _run(ms, HEVC, 8, src, [ref], p)
    assert_results_equal(got, want, "half-sample translation")
    assert (got["mvx"] == 2).all() and (got["mvy"] == 0).all()
    assert (got["satd"] == 0).all()


@pytest.mark.parametrize("d", [(1, 0), (0, -1), (5, 3), (-7, 2), (3, -8), (8, 8), (-8, -8)])
def test_h264_integral_translation_is_found_exactly(ms, d):
    ref = grating(48, 48)
    src = shifted(ref, *d)
    got, want = _run(ms, H264, 8, src, [ref], oracle.params(H264, 26))
    assert_results_equal(got, want, f"translation {d}")
    centre = got[4]  # the middle macroblock of the 3x3 picture
    assert (centre["mvx"], centre["mvy"]) == (d[0] * 4, d[1] * 4)


# ---- the committed golden fixtures ------------------------------------------------
@pytest.mark.parametrize("name", ["h264_96x64_medium", "h264_96x64_umh", "hevc_128x96_medium",
                                  "hevc_128x96_rings_cross", "hevc_96x64_10bit"])
def test_the_gpu_reproduces_the_golden_fixtures(ms, name):
    from pathlib import Path
    z = np.load(Path(__file__).resolve().parent / "golden" / f"{name}.npz")
    codec, bd = int(z["codec"]), int(z["bit_depth"])
    p = oracle.params(codec, int(z["qp"]), **dict(eval(str(z["params"]))))
    ms.upload(900, z["src"], codec, bd, as_ref=False)
    refs = list(z["refs"])
    for i, r in enumerate(refs):
        ms.upload(901 + i, r, codec, bd, as_ref=True)
    got = ms.search(900, [901 + i for i in range(len(refs))], p)
    assert_results_equal(got, z["results"].view(capi.RESULT_DTYPE), name)


@pytest.mark.parametrize("bd,amp", [(8, 0b1001), (10, 0b1001), (8, 0), (10, 0)])
def test_every_launch_shape_gives_the_oracles_results(bd, amp):
    """A fresh context times each launch shape of a class on its first
    launches (occupancy variant, CTAs for the 32x32 and 64x64 blocks or
    none, staged 8x8 patches or cache reads, the row form where the frame
    has no AMP units): the same frame searched twice per shape, and once
    more on the chosen one, equals the oracle every time."""
    import rivet_h26x_codecs_b200 as rme
    seq = synth.make_sequence(HEVC, 320, 192, bd, 3, 77 + bd, 64, 96, 2.0)
    p = oracle.params(HEVC, 30, hevc_search_range=40, hevc_search_rings=1, hevc_amp=amp)
    want = oracle.frame_search(HEVC, bd, seq.frames[2], [seq.frames[1], seq.frames[0]], p)
    with rme.MotionSearch(0) as ms2:
        for i, f in enumerate(seq.frames):
            ms2.upload(i, f, HEVC, bd, as_ref=True)
        for k in range(2 * 8 + 1):
            got = ms2.search(2, [1, 0], p)
            assert_results_equal(got, want, f"launch {k}")


@pytest.mark.parametrize("bd", [8, 10])
def test_row_form_batch_of_frames_of_two_sizes(bd):
    """A latency launch of three frames (two sizes, one and two references,
    the 16x16 level left out of one): in the row form the frames' rows are
    interleaved in the queues; each frame equals the oracle."""
    import rivet_h26x_codecs_b200 as rme
    a = synth.make_sequence(HEVC, 256, 160, bd, 3, 31 + bd, 48, 64, 2.0).frames
    b = synth.make_sequence(HEVC, 192, 128, bd, 2, 41 + bd, 48, 64, 2.0).frames
    pa = oracle.params(HEVC, 32, hevc_search_range=32)
    pb = oracle.params(HEVC, 28, hevc_search_range=24, hevc_pu_mask=0b1101)
    wants = [oracle.frame_search(HEVC, bd, a[2], [a[1], a[0]], pa),
             oracle.frame_search(HEVC, bd, a[1], [a[0]], pa),
             oracle.frame_search(HEVC, bd, b[1], [b[0]], pb)]
    with rme.MotionSearch(0) as ms2:
        for i, f in enumerate(a):
            ms2.upload(i, f, HEVC, bd, as_ref=True)
        for i, f in enumerate(b):
            ms2.upload(10 + i, f, HEVC, bd, as_ref=True)
        for k in range(3):
            got = ms2.search_batch([(2, [1, 0]), (1, [0]), (11, [10])], [pa, pa, pb])
            for j, (g, w) in enumerate(zip(got, wants)):
                assert_results_equal(g, w, f"launch {k} frame {j}")
