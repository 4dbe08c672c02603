"""Seeded synthetic video for the motion-search workloads.

The reference measures its encoders on real clips; no dataset is available
here, so sequences are generated the way the workload definitions describe
them: a source picture that is a sum of eight random 2-D sinusoids
(periods 4-64 px, amplitudes 4-40) plus uniform integer noise in +-6 about
mean 128, then each following picture is the previous one moved by a
seeded quarter-sample vector per block — formed with the codec's own
interpolation (H.264 6-tap / bilinear average per 8.4.2.2.1, HEVC 8-tap
uni-prediction per 8.5.3.3.3) — plus rounded Gaussian noise. Generation is
host-side numpy; the same bytes feed the CUDA library and the oracle, so
no floating-point detail here can affect parity.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

H264, HEVC = 0, 1

QPEL_FILTERS = np.array([[0, 0, 0, 0, 0, 0, 0, 0],
                         [-1, 4, -10, 58, 17, -5, 1, 0],
                         [-1, 4, -11, 40, 40, -11, 4, -1],
                         [0, 1, -5, 17, 58, -10, 4, -1]], dtype=np.int64)


def seed_for(config: int, stream: int = 0) -> int:
    return 0x5EED0000 + 1000 * config + stream


def source_picture(rng: np.random.Generator, w: int, h: int, bit_depth: int) -> np.ndarray:
    """Sum of 8 sinusoids + uniform noise in [-6, 6], mean 128, clamped."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    acc = np.zeros((h, w), np.float64)
    for _ in range(8):
        period = rng.uniform(4.0, 64.0)
        amp = rng.uniform(4.0, 40.0)
        theta = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        acc += amp * np.cos(2.0 * np.pi * (xx * np.cos(theta) + yy * np.sin(theta)) / period + phase)
    acc += rng.integers(-6, 7, size=(h, w))
    acc = np.floor(acc - acc.mean() + 128.0 + 0.5)
    pic = np.clip(acc, 0, 255)
    if bit_depth > 8:
        pic = np.clip(pic * (1 << (bit_depth - 8)), 0, (1 << bit_depth) - 1)
    return pic.astype(np.uint8 if bit_depth == 8 else np.uint16)


def _tap6(a, b, c, d, e, f):
    return a + f - 5 * (b + e) + 20 * (c + d)


def h264_half_planes(p: np.ndarray, maxv: int):
    """G, b, h, j of an edge-padded int64 plane (valid away from the edge)."""
    g = p
    b = np.zeros_like(g)
    b[:, 2:-3] = np.clip((_tap6(g[:, :-5], g[:, 1:-4], g[:, 2:-3], g[:, 3:-2], g[:, 4:-1], g[:, 5:]) + 16) >> 5,
                         0, maxv)
    inter = np.zeros_like(g)
    inter[2:-3, :] = _tap6(g[:-5], g[1:-4], g[2:-3], g[3:-2], g[4:-1], g[5:])
    hh = np.clip((inter + 16) >> 5, 0, maxv)
    j = np.zeros_like(g)
    j[:, 2:-3] = np.clip((_tap6(inter[:, :-5], inter[:, 1:-4], inter[:, 2:-3], inter[:, 3:-2], inter[:, 4:-1],
                                inter[:, 5:]) + 512) >> 10, 0, maxv)
    return g, b, hh, j


# (plane, dx, dy, plane2, dx2, dy2) per quarter fraction, 8.4.2.2.1
_H264_QPEL = [(0, 0, 0, -1, 0, 0), (0, 0, 0, 1, 0, 0), (1, 0, 0, -1, 0, 0), (1, 0, 0, 0, 1, 0),
              (0, 0, 0, 2, 0, 0), (1, 0, 0, 2, 0, 0), (1, 0, 0, 3, 0, 0), (1, 0, 0, 2, 1, 0),
              (2, 0, 0, -1, 0, 0), (2, 0, 0, 3, 0, 0), (3, 0, 0, -1, 0, 0), (3, 0, 0, 2, 1, 0),
              (2, 0, 0, 0, 0, 1), (2, 0, 0, 1, 0, 1), (3, 0, 0, 1, 0, 1), (2, 1, 0, 1, 0, 1)]


def warp_h264(prev: np.ndarray, mvs: np.ndarray, block: int, maxv: int) -> np.ndarray:
    """Each block x block region moved by mvs[by, bx] (quarter samples)."""
    h, w = prev.shape
    m = int(np.abs(mvs).max()) // 4 + 8
    pp = np.pad(prev.astype(np.int64), m, mode="edge")
    planes = h264_half_planes(pp, maxv)
    out = np.empty_like(prev)
    for by in range(mvs.shape[0]):
        for bx in range(mvs.shape[1]):
            qx, qy = int(mvs[by, bx, 0]), int(mvs[by, bx, 1])
            y0, x0 = by * block, bx * block
            bh, bw = min(block, h - y0), min(block, w - x0)
            xi, yi = x0 + (qx >> 2) + m, y0 + (qy >> 2) + m
            p1, dx1, dy1, p2, dx2, dy2 = _H264_QPEL[(qy & 3) * 4 + (qx & 3)]
            a = planes[p1][yi + dy1:yi + dy1 + bh, xi + dx1:xi + dx1 + bw]
            if p2 >= 0:
                b = planes[p2][yi + dy2:yi + dy2 + bh, xi + dx2:xi + dx2 + bw]
                a = (a + b + 1) >> 1
            out[y0:y0 + bh, x0:x0 + bw] = a
    return out


def warp_hevc(prev: np.ndarray, mvs: np.ndarray, block: int, bit_depth: int) -> np.ndarray:
    """Each region moved by its quarter-sample vector through HEVC luma
    uni-prediction (8-tap, shift1 = BitDepth - 8, >> 6, uni rounding)."""
    h, w = prev.shape
    m = int(np.abs(mvs).max()) // 4 + 8
    pp = np.pad(prev.astype(np.int64), m, mode="edge")
    shift1, shift3, maxv = bit_depth - 8, 14 - bit_depth, (1 << bit_depth) - 1
    out = np.empty_like(prev)
    for by in range(mvs.shape[0]):
        for bx in range(mvs.shape[1]):
            qx, qy = int(mvs[by, bx, 0]), int(mvs[by, bx, 1])
            y0, x0 = by * block, bx * block
            bh, bw = min(block, h - y0), min(block, w - x0)
            xi, yi = x0 + (qx >> 2) + m, y0 + (qy >> 2) + m
            fx, fy = qx & 3, qy & 3
            win = pp[yi - 3:yi + bh + 4, xi - 3:xi + bw + 4]
            if fx == 0 and fy == 0:
                p14 = win[3:3 + bh, 3:3 + bw] << shift3
            elif fy == 0:
                f = QPEL_FILTERS[fx]
                p14 = sum(f[k] * win[3:3 + bh, k:k + bw] for k in range(8)) >> shift1
            elif fx == 0:
                f = QPEL_FILTERS[fy]
                p14 = sum(f[k] * win[k:k + bh, 3:3 + bw] for k in range(8)) >> shift1
            else:
                fh, fv = QPEL_FILTERS[fx], QPEL_FILTERS[fy]
                tmp = sum(fh[k] * win[:, k:k + bw] for k in range(8)) >> shift1
                tmp = tmp.astype(np.int16).astype(np.int64)
                p14 = sum(fv[k] * tmp[k:k + bh] for k in range(8)) >> 6
            p14 = p14.astype(np.int16).astype(np.int64)
            out[y0:y0 + bh, x0:x0 + bw] = np.clip((p14 + (1 << (shift3 - 1))) >> shift3, 0, maxv)
    return out


@dataclass
class Sequence:
    codec: int
    bit_depth: int
    width: int
    height: int
    frames: list = field(default_factory=list)  # numpy pictures, frame 0 first
    seed: int = 0


def make_sequence(codec: int, width: int, height: int, bit_depth: int, nframes: int, seed: int,
                  block: int, max_q: int, sigma: float) -> Sequence:
    """nframes pictures: a sinusoid source, then warp(previous) + noise per
    frame; block motion drawn uniformly in [-max_q, max_q] quarter samples."""
    rng = np.random.default_rng(seed)
    maxv = (1 << bit_depth) - 1
    seq = Sequence(codec, bit_depth, width, height, seed=seed)
    pic = source_picture(rng, width, height, bit_depth)
    seq.frames.append(pic)
    nby, nbx = -(-height // block), -(-width // block)
    for _ in range(1, nframes):
        mvs = rng.integers(-max_q, max_q + 1, size=(nby, nbx, 2))
        moved = warp_h264(pic, mvs, block, maxv) if codec == H264 else warp_hevc(pic, mvs, block, bit_depth)
        noise = np.floor(rng.normal(0.0, sigma, size=moved.shape) + 0.5).astype(np.int64)
        pic = np.clip(moved.astype(np.int64) + noise, 0, maxv).astype(pic.dtype)
        seq.frames.append(pic)
    return seq


# The workloads: (codec, width, height, bit depth, refs, search settings).
def config0(nframes: int = 2) -> Sequence:
    """H.264 CIF 8-bit P-frame against 1 reference; 16x16 motion U[-12,12] px
    quarter-sample, sigma 2."""
    return make_sequence(H264, 352, 288, 8, nframes, seed_for(0), 16, 48, 2.0)


def config1(nframes: int = 62, width: int = 1920, height: int = 1080) -> Sequence:
    """HEVC 8-bit 1080p; 64x64 region motion U[-40,40] px quarter-sample,
    sigma 2. Frame t >= 2 searches frames t-1 and t-2."""
    return make_sequence(HEVC, width, height, 8, nframes, seed_for(1), 64, 160, 2.0)


def config2(nframes: int = 36, width: int = 3840, height: int = 2160) -> Sequence:
    """HEVC 10-bit 2160p; 64x64 region motion U[-96,96] px, sigma 6."""
    return make_sequence(HEVC, width, height, 10, nframes, seed_for(2), 64, 384, 6.0)


def stream_sequence(codec: int, width: int, height: int, bit_depth: int, nframes: int, stream: int,
                    config: int = 3) -> Sequence:
    """One stream of the mixed workloads, with its own seed."""
    block = 16 if codec == H264 else 64
    max_q = 48 if codec == H264 else 160
    sigma = 6.0 if bit_depth > 8 else 2.0
    return make_sequence(codec, width, height, bit_depth, nframes, seed_for(config, stream), block, max_q, sigma)
