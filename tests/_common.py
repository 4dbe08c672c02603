"""Helpers shared by the tests: seeded pictures, jobs, and field-by-field
comparison of result arrays."""
from __future__ import annotations

import numpy as np

import rivet_h26x_codecs_b200.capi as capi


def lcg_picture(w: int, h: int, seed: int, bit_depth: int = 8) -> np.ndarray:
    """The reference tests' picture generator: s = s*1103515245 + 12345,
    sample = (s >> 16) (h264_hpel.rs:1037-1045, h265_search.rs:294-302),
    scaled to the depth for deeper samples."""
    out = np.zeros((h, w), np.uint8 if bit_depth == 8 else np.uint16)
    s = seed & 0xFFFFFFFF
    for y in range(h):
        for x in range(w):
            s = (s * 1103515245 + 12345) & 0xFFFFFFFF
            v = (s >> 16) & 255
            out[y, x] = v if bit_depth == 8 else (((s >> 16) & 0xFFFF) % (1 << bit_depth))
    return out


def random_picture(rng: np.random.Generator, w: int, h: int, bit_depth: int, smooth: int = 3) -> np.ndarray:
    """Textured random picture (a box-filtered noise field), so searches
    have structure to descend."""
    maxv = (1 << bit_depth) - 1
    a = rng.integers(0, maxv + 1, size=(h + 2 * smooth, w + 2 * smooth)).astype(np.float64)
    k = 2 * smooth + 1
    c = np.cumsum(np.cumsum(np.pad(a, ((1, 0), (1, 0))), 0), 1)
    box = (c[k:, k:] - c[:-k, k:] - c[k:, :-k] + c[:-k, :-k]) / (k * k)
    box = box[:h, :w]
    out = np.clip(np.floor(box + rng.normal(0, maxv / 64, size=box.shape)), 0, maxv)
    return out.astype(np.uint8 if bit_depth == 8 else np.uint16)


def shifted(pic: np.ndarray, dx: int, dy: int, rng: np.random.Generator | None = None, noise: float = 0.0):
    """pic translated so that a block at p equals the reference at p + (dx, dy)
    (edge-clamped), with optional rounded Gaussian noise."""
    h, w = pic.shape
    ys = np.clip(np.arange(h) + dy, 0, h - 1)
    xs = np.clip(np.arange(w) + dx, 0, w - 1)
    out = pic[ys][:, xs].astype(np.int64)
    if rng is not None and noise > 0:
        out += np.floor(rng.normal(0, noise, size=out.shape) + 0.5).astype(np.int64)
    maxv = 255 if pic.dtype == np.uint8 else 65535
    return np.ascontiguousarray(np.clip(out, 0, maxv).astype(pic.dtype))


def random_jobs(rng: np.random.Generator, codec: int, w: int, h: int, nref: int, n: int,
                sizes=((8, 8), (16, 16), (16, 8), (8, 16), (32, 32), (64, 64), (4, 4), (8, 4), (4, 8), (32, 16),
                       (16, 64), (64, 16), (12, 16), (16, 12), (64, 48), (48, 64), (32, 24), (24, 32), (32, 8),
                       (8, 32)),
                spread: int = 120) -> np.ndarray:
    jobs = np.zeros(n, capi.JOB_DTYPE)
    max_seeds = 8 if codec == capi.RME_CODEC_H264 else capi.RME_MAX_SEEDS
    for i in range(n):
        bw, bh = sizes[rng.integers(len(sizes))]
        bw, bh = min(bw, w), min(bh, h)
        jobs[i]["x"] = rng.integers(0, (w - bw) // 4 + 1) * 4
        jobs[i]["y"] = rng.integers(0, (h - bh) // 4 + 1) * 4
        jobs[i]["w"], jobs[i]["h"] = bw, bh
        jobs[i]["ref"] = rng.integers(nref)
        ns = rng.integers(0, max_seeds + 1)
        jobs[i]["nseeds"] = ns
        jobs[i]["mvp"] = rng.integers(-spread, spread + 1, size=(2, 2))
        seeds = rng.integers(-spread, spread + 1, size=(capi.RME_MAX_SEEDS, 2))
        if ns > 2:  # repeat some seeds, as encoders' candidate lists do
            seeds[ns - 1] = seeds[0]
        jobs[i]["seeds"] = seeds
        jobs[i]["flags"] = capi.RME_JOB_SCORE_ONLY if (codec == capi.RME_CODEC_H264 and rng.random() < 0.2) else 0
    return jobs


def assert_results_equal(got: np.ndarray, want: np.ndarray, what: str = "") -> None:
    assert got.shape == want.shape, f"{what}: {got.shape} vs {want.shape}"
    for name in capi.RESULT_DTYPE.names:
        bad = np.nonzero(got[name] != want[name])[0]
        if len(bad):
            i = bad[0]
            raise AssertionError(f"{what}: field {name} differs at {len(bad)} of {len(got)} results; "
                                 f"first index {i}: got {got[i]} want {want[i]}")
