// The lookahead's motion estimation at half resolution, for the HEVC
// encoder's quantiser propagation (encode/h265_cutree.rs) and the H.264
// encoder's (encode/h264_lookahead.rs): the half-resolution plane of a
// picture and its blocks' intra costs, the per-block motion search against
// a reference and the SATD against the average of two displaced blocks.
//
// The search reads the left and above blocks' vectors as seeds, so its
// blocks form a wavefront. Warps claim blocks in anti-diagonal order from
// one counter and wait (bounded) for the two blocks they read: every block
// a warp waits for was claimed earlier by a running warp, so the wait
// always ends unless a wait bound runs out, which sets the status word.
#include <cuda_runtime.h>

#include "rme_internal.h"

namespace rme {
namespace {

constexpr unsigned kAll = 0xffffffffu;

// LowRes::new (h265_cutree.rs:61-110): the 2x2 mean of the picture
// (clamped at its edges) shifted to 8 bits, over whole 8x8 blocks, the
// border replicated: every padded position is the value of its clamped
// position.
template <class S>
__global__ void lowres_build_kernel(const S* __restrict__ pic, int pstride, int w, int h, int bd, LowresDesc L) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
  const int rows = L.ph + 2 * kLowresPad;
  if (X >= L.stride || Y >= rows) return;
  const int lw = (w + 1) / 2, lh = (h + 1) / 2;
  const int xx = min(max(X - kLowresPad, 0), L.pw - 1), yy = min(max(Y - kLowresPad, 0), L.ph - 1);
  const int x2 = 2 * min(xx, lw - 1), y2 = 2 * min(yy, lh - 1);
  auto at = [&](int x, int y) { return (int)pic[(ptrdiff_t)min(y, h - 1) * pstride + min(x, w - 1)]; };
  const int s = at(x2, y2) + at(x2 + 1, y2) + at(x2, y2 + 1) + at(x2 + 1, y2 + 1);
  L.plane[(ptrdiff_t)Y * L.stride + X] = (uint8_t)min(((s + 2) >> 2) >> (bd - 8), 255);
}

// One 4x4 tile's Hadamard SATD, (sum + 1) >> 1 (dsp/distortion.rs:350-381).
template <class S>
__device__ __forceinline__ uint32_t satd4x4_tile(const S* a, int as, const S* b, int bs) {
  int d[16];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) d[r * 4 + c] = (int)a[(ptrdiff_t)r * as + c] - (int)b[(ptrdiff_t)r * bs + c];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int p = d[i * 4], q = d[i * 4 + 1], u = d[i * 4 + 2], v = d[i * 4 + 3];
    const int s0 = p + v, s1 = q + u, s2 = q - u, s3 = p - v;
    d[i * 4] = s0 + s1;
    d[i * 4 + 1] = s3 + s2;
    d[i * 4 + 2] = s0 - s1;
    d[i * 4 + 3] = s3 - s2;
  }
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int p = d[j], q = d[4 + j], u = d[8 + j], v = d[12 + j];
    const int s0 = p + v, s1 = q + u, s2 = q - u, s3 = p - v;
    sum += abs(s0 + s1) + abs(s3 + s2) + abs(s0 - s1) + abs(s3 - s2);
  }
  return (sum + 1) >> 1;
}

template <class S>
__device__ uint32_t satd8x8(const S* a, int as, const S* b, int bs) {
  uint32_t total = 0;
  for (int ty = 0; ty < 2; ++ty)
    for (int tx = 0; tx < 2; ++tx)
      total += satd4x4_tile<S>(a + (ptrdiff_t)(ty * 4) * as + tx * 4, as, b + (ptrdiff_t)(ty * 4) * bs + tx * 4, bs);
  return total;
}

// intra_cost (h265_cutree.rs:118-140), one thread per block: the least SATD
// of the flat, horizontal and vertical predictions from the samples above
// and left, floored at 16.
__global__ void lowres_intra_kernel(LowresDesc L) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= L.bw * L.bh) return;
  const int x = (b % L.bw) * 8, y = (b / L.bw) * 8;
  const uint8_t* src = L.plane + (ptrdiff_t)(y + kLowresPad) * L.stride + x + kLowresPad;
  uint8_t top[8], left[8];
  int st = 0;
  for (int i = 0; i < 8; ++i) {
    top[i] = src[i - L.stride];
    left[i] = src[(ptrdiff_t)i * L.stride - 1];
    st += top[i] + left[i];
  }
  uint8_t pred[64];
  const uint8_t dc = (uint8_t)((st + 8) / 16);
  for (int i = 0; i < 64; ++i) pred[i] = dc;
  uint32_t best = satd8x8<uint8_t>(src, L.stride, pred, 8);
  for (int i = 0; i < 64; ++i) pred[i] = left[i / 8];
  best = min(best, satd8x8<uint8_t>(src, L.stride, pred, 8));
  for (int i = 0; i < 64; ++i) pred[i] = top[i % 8];
  best = min(best, satd8x8<uint8_t>(src, L.stride, pred, 8));
  L.intra[b] = max(best, 16u);
}

__device__ __forceinline__ uint32_t ld_acquire32(const int32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release32(int32_t* p, int32_t v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// A bounded wait (lane 0) for block b to be done: at most `limit` polls,
// then the status word records the timeout and the wait gives up.
__device__ __forceinline__ bool wait_done(const int32_t* done, int b, uint32_t* status, uint32_t limit = kSpinLimit) {
  uint32_t ns = 32;
  for (uint32_t it = 0; it < limit; ++it) {
    if (ld_acquire32(done + b)) return true;
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  atomicOr(status, kStatusWaitTimeout);
  return false;
}

// Eight bytes of a row at any byte address (three aligned loads).
__device__ __forceinline__ void ld8(const uint8_t* p, uint32_t& a, uint32_t& b) {
  const uintptr_t u = reinterpret_cast<uintptr_t>(p);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(u & ~uintptr_t(3));
  const uint32_t sh = (uint32_t)(u & 3) * 8u;
  const uint32_t w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2);
  a = __funnelshift_r(w0, w1, sh);
  b = __funnelshift_r(w1, w2, sh);
}

struct Pick2 {
  uint32_t cost;
  int lane;
};
__device__ __forceinline__ Pick2 argmin(uint32_t c) {
  const uint32_t m = __reduce_min_sync(kAll, c);
  return {m, __ffs(__ballot_sync(kAll, c == m)) - 1};
}

// search (h265_cutree.rs:152-216), one warp per block: four candidates per
// step (group g = lane / 8, lane sub = row), the first least cost taken when
// strictly below the best, as the reference's in-order scoring.
__global__ void __launch_bounds__(256) lowres_search_kernel(const LowresDesc* pairs, int npairs, const int32_t* order,
                                                            int32_t* done_all, unsigned long long* counter,
                                                            uint32_t* status, uint32_t* cost_all, rme_mv* mv_all,
                                                            uint32_t* nsad_all) {
  const int lane = threadIdx.x & 31, g = lane >> 3, sub = lane & 7;
  const int n = pairs[0].bw * pairs[0].bh, lim = kLowresPad - 1;
  for (;;) {
    unsigned long long i = 0;
    if (lane == 0) i = atomicAdd(counter, 1ull);
    i = __shfl_sync(kAll, i, 0);
    if (i >= (unsigned long long)n * npairs) break;
    // Claims interleave the pairs in wavefront order: entry e of pair pi is
    // claim e * npairs + pi, after every block it reads.
    const int pi = (int)(i % npairs), e = (int)(i / npairs);
    const LowresDesc cur = pairs[2 * pi], ref = pairs[2 * pi + 1];
    int32_t* done = done_all + (size_t)pi * n;
    uint32_t* cost = cost_all + (size_t)pi * n;
    rme_mv* mv = mv_all + (size_t)pi * n;
    uint32_t* nsad_out = nsad_all ? nsad_all + (size_t)pi * n : nullptr;
    const int packed = __ldg(order + e), bx = packed & 0xffff, by = packed >> 16, b = by * cur.bw + bx;
    if (lane == 0) {
      if (bx > 0) wait_done(done, b - 1, status);
      if (by > 0) wait_done(done, b - cur.bw, status);
    }
    __syncwarp();
    const int x = bx * 8, y = by * 8;
    const uint8_t* src = cur.plane + (ptrdiff_t)(y + kLowresPad) * cur.stride + x + kLowresPad;
    const uint8_t* rb = ref.plane + (ptrdiff_t)(y + kLowresPad) * ref.stride + x + kLowresPad;
    // This lane's source row (8-byte aligned: x, the pad and the stride
    // are multiples of 8).
    const uint32_t s0 = *reinterpret_cast<const uint32_t*>(src + (ptrdiff_t)sub * cur.stride);
    const uint32_t s1 = *reinterpret_cast<const uint32_t*>(src + (ptrdiff_t)sub * cur.stride + 4);
    auto inplane = [&](int dx, int dy) {
      return x + dx >= -lim && y + dy >= -lim && x + dx + 8 <= ref.pw + lim && y + dy + 8 <= ref.ph + lim;
    };
    auto score = [&](bool ok, int dx, int dy) -> uint32_t {
      uint32_t part = 0;
      if (ok) {
        uint32_t a, c;
        ld8(rb + (ptrdiff_t)(dy + sub) * ref.stride + dx, a, c);
        part = __vsadu4(s0, a) + __vsadu4(s1, c);
      }
      part += __shfl_xor_sync(kAll, part, 4);
      part += __shfl_xor_sync(kAll, part, 2);
      part += __shfl_xor_sync(kAll, part, 1);
      return ok ? part + 2u * (uint32_t)min(abs(dx) + abs(dy), 32) : 0xffffffffu;
    };
    // Seeds: zero, the left block's vector, the above block's.
    uint32_t lv = 0, av = 0;
    if (bx > 0) lv = __ldcg(reinterpret_cast<const unsigned int*>(mv + b - 1));
    if (by > 0) av = __ldcg(reinterpret_cast<const unsigned int*>(mv + b - cur.bw));
    const int ns = 1 + (bx > 0) + (by > 0);
    const uint32_t sv = g == 0 ? 0u : g == 1 ? (bx > 0 ? lv : av) : av;
    int dx = (int)(int16_t)(sv & 0xffffu), dy = (int)(int16_t)(sv >> 16);
    bool ok = g < ns && inplane(dx, dy);
    uint32_t nsad = __popc(__ballot_sync(kAll, ok && sub == 0));
    Pick2 p = argmin(score(ok, dx, dy));
    uint32_t bc = p.cost;
    int bxm = __shfl_sync(kAll, dx, p.lane), bym = __shfl_sync(kAll, dy, p.lane);
    if (bc == 0xffffffffu) bxm = bym = 0;  // no seed in the plane
    const int cx = bxm, cy = bym;
    for (int step = 4; step >= 1; step >>= 1) {
      for (;;) {
        dx = bxm + (g == 0 ? step : g == 1 ? -step : 0);
        dy = bym + (g == 2 ? step : g == 3 ? -step : 0);
        ok = abs(dx - cx) <= kLowresRange && abs(dy - cy) <= kLowresRange && inplane(dx, dy);
        nsad += __popc(__ballot_sync(kAll, ok && sub == 0));
        p = argmin(score(ok, dx, dy));
        if (!(p.cost < bc)) break;
        bc = p.cost;
        bxm = __shfl_sync(kAll, dx, p.lane);
        bym = __shfl_sync(kAll, dy, p.lane);
      }
    }
    // The winner's SATD: tile `lane` of the four (lanes 0..3).
    uint32_t sat = 0;
    if (lane < 4) {
      const int tx = lane & 1, ty = lane >> 1;
      sat = satd4x4_tile<uint8_t>(src + (ptrdiff_t)(ty * 4) * cur.stride + tx * 4, cur.stride,
                                  rb + (ptrdiff_t)(bym + ty * 4) * ref.stride + bxm + tx * 4, ref.stride);
    }
    sat += __shfl_xor_sync(kAll, sat, 1);
    sat += __shfl_xor_sync(kAll, sat, 2);
    if (lane == 0) {
      cost[b] = sat;
      mv[b].x = (int16_t)bxm;
      mv[b].y = (int16_t)bym;
      if (nsad_out) nsad_out[b] = nsad;
      __threadfence();
      st_release32(done + b, 1);
    }
    __syncwarp();
  }
}

// bi_cost (h265_cutree.rs:222-243), one thread per block.
__global__ void lowres_bi_kernel(LowresDesc cur, LowresDesc r0, LowresDesc r1, const rme_mv* m0, const rme_mv* m1,
                                 uint32_t* cost) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= cur.bw * cur.bh) return;
  const int x = (b % cur.bw) * 8, y = (b / cur.bw) * 8;
  const uint8_t* a = r0.plane + (ptrdiff_t)(y + m0[b].y + kLowresPad) * r0.stride + x + m0[b].x + kLowresPad;
  const uint8_t* c = r1.plane + (ptrdiff_t)(y + m1[b].y + kLowresPad) * r1.stride + x + m1[b].x + kLowresPad;
  uint8_t pred[64];
  for (int yy = 0; yy < 8; ++yy)
    for (int xx = 0; xx < 8; ++xx)
      pred[yy * 8 + xx] = (uint8_t)(((int)a[(ptrdiff_t)yy * r0.stride + xx] + c[(ptrdiff_t)yy * r1.stride + xx] + 1) >> 1);
  cost[b] = satd8x8<uint8_t>(cur.plane + (ptrdiff_t)(y + kLowresPad) * cur.stride + x + kLowresPad, cur.stride, pred, 8);
}

// ---- H.264 (h264_lookahead.rs) ----------------------------------------------

// Lookahead::add (h264_lookahead.rs:87-117): over the macroblock grid (8
// samples per macroblock), each sample the rounded mean of the picture's
// 2x2 square at (2x, 2y), its columns and rows clamped to the picture; the
// border replicated (every padded position takes its clamped position's
// value).
template <class S>
__global__ void lowres_build_h264_kernel(const S* __restrict__ pic, int pstride, int w, int h, LowresDesc L) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
  const int rows = L.ph + 2 * kLowresPad;
  if (X >= L.stride || Y >= rows) return;
  const int xx = min(max(X - kLowresPad, 0), L.pw - 1), yy = min(max(Y - kLowresPad, 0), L.ph - 1);
  const int x0 = min(2 * xx, w - 1), x1 = min(2 * xx + 1, w - 1);
  const S* r0 = pic + (ptrdiff_t)min(2 * yy, h - 1) * pstride;
  const S* r1 = pic + (ptrdiff_t)min(2 * yy + 1, h - 1) * pstride;
  const int s = (int)r0[x0] + r0[x1] + r1[x0] + r1[x1];
  reinterpret_cast<S*>(L.plane)[(ptrdiff_t)Y * L.stride + X] = (S)((s + 2) >> 2);
}

// intra_costs (h264_lookahead.rs:146-222), one thread per block: DC from
// the neighbours there are (the block's own mean with none), vertical where
// there is a row above, horizontal where there is a column to the left, the
// bilinear blend of both edges where both are; the least SATD, plus 12.
template <class S>
__global__ void lowres_intra_h264_kernel(LowresDesc L) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= L.bw * L.bh) return;
  const int bx = b % L.bw, by = b / L.bw;
  const S* src = reinterpret_cast<const S*>(L.plane) + (ptrdiff_t)(by * 8 + kLowresPad) * L.stride + bx * 8 + kLowresPad;
  const bool ht = by > 0, hl = bx > 0;
  int t[8], l[8], st = 0, sl = 0;
  for (int i = 0; i < 8; ++i) {
    t[i] = src[i - L.stride];
    l[i] = src[(ptrdiff_t)i * L.stride - 1];
    st += t[i];
    sl += l[i];
  }
  int dc;
  if (ht && hl) {
    dc = (st + sl + 8) >> 4;
  } else if (ht || hl) {
    dc = ((ht ? st : sl) + 4) >> 3;
  } else {
    int sum = 0;
    for (int yy = 0; yy < 8; ++yy)
      for (int xx = 0; xx < 8; ++xx) sum += src[(ptrdiff_t)yy * L.stride + xx];
    dc = (sum + 32) >> 6;
  }
  S pred[64];
  for (int i = 0; i < 64; ++i) pred[i] = (S)dc;
  uint32_t best = satd8x8<S>(src, L.stride, pred, 8);
  if (ht) {
    for (int i = 0; i < 64; ++i) pred[i] = (S)t[i & 7];
    best = min(best, satd8x8<S>(src, L.stride, pred, 8));
  }
  if (hl) {
    for (int i = 0; i < 64; ++i) pred[i] = (S)l[i >> 3];
    best = min(best, satd8x8<S>(src, L.stride, pred, 8));
  }
  if (ht && hl) {
    for (int yy = 0; yy < 8; ++yy)
      for (int xx = 0; xx < 8; ++xx)
        pred[yy * 8 + xx] = (S)((t[xx] * (8 - yy) + l[yy] * (8 - xx) + t[7] * yy + l[7] * xx + 8) >> 4);
    best = min(best, satd8x8<S>(src, L.stride, pred, 8));
  }
  L.intra[b] = best + 12;
}

// One row of 8 samples at any sample address, as 32-bit words (two for u8,
// four for u16), from aligned loads.
template <class S>
struct Row8;
template <>
struct Row8<uint8_t> {
  uint32_t w[2];
  __device__ __forceinline__ void load(const uint8_t* p) {
    uint32_t a, b;
    ld8(p, a, b);
    w[0] = a;
    w[1] = b;
  }
  __device__ __forceinline__ uint32_t sad(const Row8& o) const { return __vsadu4(w[0], o.w[0]) + __vsadu4(w[1], o.w[1]); }
};
template <>
struct Row8<uint16_t> {
  uint32_t w[4];
  __device__ __forceinline__ void load(const uint16_t* p) {
    const uintptr_t u = reinterpret_cast<uintptr_t>(p);
    const uint32_t* q = reinterpret_cast<const uint32_t*>(u & ~uintptr_t(3));
    const uint32_t sh = (uint32_t)(u & 3) * 8u;
    uint32_t v[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) v[i] = __ldg(q + i);
#pragma unroll
    for (int i = 0; i < 4; ++i) w[i] = __funnelshift_r(v[i], v[i + 1], sh);
  }
  __device__ __forceinline__ uint32_t sad(const Row8& o) const {
    return __vsadu2(w[0], o.w[0]) + __vsadu2(w[1], o.w[1]) + __vsadu2(w[2], o.w[2]) + __vsadu2(w[3], o.w[3]);
  }
};

// search (h264_lookahead.rs:227-376), one warp per block, eight points per
// pass (group g = lane / 4 scores one point, lane q = lane % 4 its rows q
// and q + 4). The window is the reference's: 16 samples into the border,
// at most 32 from the block. From the zero vector, the left and above
// blocks' vectors (zero where there is no such block) clamped to the window,
// each scored unless it is the best's point, then the hexagon (after a step
// in direction k only k - 1, k and k + 1 are new), at most 16 steps, then
// the eight-point square; the SAD + 2 * min(|mx| + |my|, 64) of each point,
// the first least cost taken when strictly below the best (the reference's
// in-order scoring), the winner's SATD.
template <class S>
__global__ void __launch_bounds__(256) lowres_search_h264_kernel(const LowresDesc* pairs, int npairs,
                                                                 const int32_t* order, int32_t* done_all,
                                                                 unsigned long long* counter, uint32_t* status,
                                                                 uint32_t* cost_all, rme_mv* mv_all,
                                                                 uint32_t* nsad_all) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int n = pairs[0].bw * pairs[0].bh, lim = kLowresPad - 8;
  for (;;) {
    unsigned long long i = 0;
    if (lane == 0) i = atomicAdd(counter, 1ull);
    i = __shfl_sync(kAll, i, 0);
    if (i >= (unsigned long long)n * npairs) break;
    const int pi = (int)(i % npairs), e = (int)(i / npairs);  // as lowres_search_kernel's claims
    const LowresDesc cur = pairs[2 * pi], ref = pairs[2 * pi + 1];
    const S* cplane = reinterpret_cast<const S*>(cur.plane);
    const S* rplane = reinterpret_cast<const S*>(ref.plane);
    int32_t* done = done_all + (size_t)pi * n;
    uint32_t* cost = cost_all + (size_t)pi * n;
    rme_mv* mv = mv_all + (size_t)pi * n;
    uint32_t* nsad_out = nsad_all ? nsad_all + (size_t)pi * n : nullptr;
    const int packed = __ldg(order + e), bx = packed & 0xffff, by = packed >> 16, b = by * cur.bw + bx;
    if (lane == 0) {
      if (bx > 0) wait_done(done, b - 1, status);
      if (by > 0) wait_done(done, b - cur.bw, status);
    }
    __syncwarp();
    const int x = bx * 8, y = by * 8;
    const S* src = cplane + (ptrdiff_t)(y + kLowresPad) * cur.stride + x + kLowresPad;
    const S* rb = rplane + (ptrdiff_t)(y + kLowresPad) * ref.stride + x + kLowresPad;
    const int lx = max(-x - lim, -2 * kLowresRange), hx = min(cur.pw - 8 - x + lim, 2 * kLowresRange);
    const int ly = max(-y - lim, -2 * kLowresRange), hy = min(cur.ph - 8 - y + lim, 2 * kLowresRange);
    // This lane's two source rows (aligned: x, the pad and the stride are
    // multiples of 8 samples).
    Row8<S> s0, s1;
    s0.load(src + (ptrdiff_t)q * cur.stride);
    s1.load(src + (ptrdiff_t)(q + 4) * cur.stride);
    auto score = [&](bool ok, int dx, int dy) -> uint32_t {
      uint32_t part = 0;
      if (ok) {
        Row8<S> a, c;
        a.load(rb + (ptrdiff_t)(dy + q) * ref.stride + dx);
        c.load(rb + (ptrdiff_t)(dy + q + 4) * ref.stride + dx);
        part = s0.sad(a) + s1.sad(c);
      }
      part += __shfl_xor_sync(kAll, part, 2);
      part += __shfl_xor_sync(kAll, part, 1);
      return ok ? part + 2u * (uint32_t)min(abs(dx) + abs(dy), 64) : 0xffffffffu;
    };
    auto inwin = [&](int dx, int dy) { return dx >= lx && dx <= hx && dy >= ly && dy <= hy; };
    // The zero vector and the two candidates, scored at once (groups 0..2),
    // resolved in the reference's order.
    uint32_t lv = 0, av = 0;
    if (bx > 0) lv = __ldcg(reinterpret_cast<const unsigned int*>(mv + b - 1));
    if (by > 0) av = __ldcg(reinterpret_cast<const unsigned int*>(mv + b - cur.bw));
    const int c0x = min(max((int)(int16_t)(lv & 0xffffu), lx), hx), c0y = min(max((int)(int16_t)(lv >> 16), ly), hy);
    const int c1x = min(max((int)(int16_t)(av & 0xffffu), lx), hx), c1y = min(max((int)(int16_t)(av >> 16), ly), hy);
    int dx = g == 1 ? c0x : g == 2 ? c1x : 0, dy = g == 1 ? c0y : g == 2 ? c1y : 0;
    const uint32_t sc = score(g < 3, dx, dy);
    const uint32_t z = __shfl_sync(kAll, sc, 0), k0 = __shfl_sync(kAll, sc, 4), k1 = __shfl_sync(kAll, sc, 8);
    uint32_t bc = z, nsad = 1;
    int bxm = 0, bym = 0;
    if (c0x != 0 || c0y != 0) {
      ++nsad;
      if (k0 < bc) {
        bc = k0;
        bxm = c0x;
        bym = c0y;
      }
    }
    if (c1x != bxm || c1y != bym) {
      ++nsad;
      if (k1 < bc) {
        bc = k1;
        bxm = c1x;
        bym = c1y;
      }
    }
    // The hexagon, its points in order around it.
    const int hxo = g == 0 ? -2 : g == 1 ? -1 : g == 2 ? 1 : g == 3 ? 2 : g == 4 ? 1 : -1;
    const int hyo = g == 0 ? 0 : g < 3 ? -2 : g == 3 ? 0 : 2;
    int from = -1;
    for (int it = 0; it < kLowresRange; ++it) {
      uint32_t live = 0x3f;
      if (from >= 0) {
        const uint32_t r = 7u << (from + 5);
        live = (r | r >> 6 | r >> 12) & 0x3f;
      }
      dx = bxm + hxo;
      dy = bym + hyo;
      const bool ok = g < 6 && ((live >> g) & 1) && inwin(dx, dy);
      nsad += __popc(__ballot_sync(kAll, ok && q == 0));
      const Pick2 p = argmin(score(ok, dx, dy));
      if (!(p.cost < bc)) break;
      bc = p.cost;
      bxm = __shfl_sync(kAll, dx, p.lane);
      bym = __shfl_sync(kAll, dy, p.lane);
      from = p.lane >> 2;
    }
    // The square around the hexagon's centre.
    {
      const int k = g < 4 ? g : g + 1;  // the 3x3 square without its centre
      dx = bxm + k % 3 - 1;
      dy = bym + k / 3 - 1;
      const bool ok = inwin(dx, dy);
      nsad += __popc(__ballot_sync(kAll, ok && q == 0));
      const Pick2 p = argmin(score(ok, dx, dy));
      if (p.cost < bc) {
        bc = p.cost;
        bxm = __shfl_sync(kAll, dx, p.lane);
        bym = __shfl_sync(kAll, dy, p.lane);
      }
    }
    // The winner's SATD: tile `lane` of the four (lanes 0..3).
    uint32_t sat = 0;
    if (lane < 4) {
      const int tx = lane & 1, ty = lane >> 1;
      sat = satd4x4_tile<S>(src + (ptrdiff_t)(ty * 4) * cur.stride + tx * 4, cur.stride,
                            rb + (ptrdiff_t)(bym + ty * 4) * ref.stride + bxm + tx * 4, ref.stride);
    }
    sat += __shfl_xor_sync(kAll, sat, 1);
    sat += __shfl_xor_sync(kAll, sat, 2);
    if (lane == 0) {
      cost[b] = sat;
      mv[b].x = (int16_t)bxm;
      mv[b].y = (int16_t)bym;
      if (nsad_out) nsad_out[b] = nsad;
      __threadfence();
      st_release32(done + b, 1);
    }
    __syncwarp();
  }
}

// The average-of-two cost of estimate() (h264_lookahead.rs:417-432), one
// thread per block: the SATD against the rounded average of the blocks the
// two vectors point at.
template <class S>
__global__ void lowres_bi_h264_kernel(LowresDesc cur, LowresDesc r0, LowresDesc r1, const rme_mv* m0, const rme_mv* m1,
                                      uint32_t* cost) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= cur.bw * cur.bh) return;
  const int x = (b % cur.bw) * 8, y = (b / cur.bw) * 8;
  const S* a = reinterpret_cast<const S*>(r0.plane) + (ptrdiff_t)(y + m0[b].y + kLowresPad) * r0.stride + x + m0[b].x +
               kLowresPad;
  const S* c = reinterpret_cast<const S*>(r1.plane) + (ptrdiff_t)(y + m1[b].y + kLowresPad) * r1.stride + x + m1[b].x +
               kLowresPad;
  S pred[64];
  for (int yy = 0; yy < 8; ++yy)
    for (int xx = 0; xx < 8; ++xx)
      pred[yy * 8 + xx] = (S)(((int)a[(ptrdiff_t)yy * r0.stride + xx] + c[(ptrdiff_t)yy * r1.stride + xx] + 1) >> 1);
  const S* src = reinterpret_cast<const S*>(cur.plane) + (ptrdiff_t)(y + kLowresPad) * cur.stride + x + kLowresPad;
  cost[b] = satd8x8<S>(src, cur.stride, pred, 8);
}

// The wavefront's wait on a flag nothing sets, with a short poll limit:
// the failure path of a dependency that never completes, taken on purpose.
__global__ void probe_wait_kernel(const int32_t* flag, uint32_t limit, uint32_t* status) {
  if ((threadIdx.x & 31) == 0) wait_done(flag, 0, status, limit);
}

}  // namespace

cudaError_t launch_probe_wait(const int32_t* flag, uint32_t limit, uint32_t* status, cudaStream_t s) {
  probe_wait_kernel<<<1, 32, 0, s>>>(flag, limit, status);
  return cudaGetLastError();
}

cudaError_t launch_lowres_build(const DevPlanes& pic, int bd, int w, int h, const LowresDesc& L, cudaStream_t s) {
  dim3 blk(32, 8), grd((L.stride + 31) / 32, (L.ph + 2 * kLowresPad + 7) / 8);
  if (L.h264) {
    if (bd == 8) {
      lowres_build_h264_kernel<uint8_t><<<grd, blk, 0, s>>>((const uint8_t*)pic.base + pic.origin, pic.stride, w, h, L);
      lowres_intra_h264_kernel<uint8_t><<<(L.bw * L.bh + 127) / 128, 128, 0, s>>>(L);
    } else {
      lowres_build_h264_kernel<uint16_t>
          <<<grd, blk, 0, s>>>((const uint16_t*)pic.base + pic.origin, pic.stride, w, h, L);
      lowres_intra_h264_kernel<uint16_t><<<(L.bw * L.bh + 127) / 128, 128, 0, s>>>(L);
    }
    return cudaGetLastError();
  }
  if (bd == 8)
    lowres_build_kernel<uint8_t><<<grd, blk, 0, s>>>((const uint8_t*)pic.base + pic.origin, pic.stride, w, h, bd, L);
  else
    lowres_build_kernel<uint16_t><<<grd, blk, 0, s>>>((const uint16_t*)pic.base + pic.origin, pic.stride, w, h, bd, L);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  lowres_intra_kernel<<<(L.bw * L.bh + 127) / 128, 128, 0, s>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_lowres_search(const LowresDesc* pairs, int npairs, const LowresDesc& first, const int32_t* order,
                                 int32_t* done, unsigned long long* counter, uint32_t* status, uint32_t* cost,
                                 rme_mv* mv, uint32_t* nsad, int grid, cudaStream_t s) {
  if (!first.h264)
    lowres_search_kernel<<<grid, 256, 0, s>>>(pairs, npairs, order, done, counter, status, cost, mv, nsad);
  else if (first.bytes == 1)
    lowres_search_h264_kernel<uint8_t>
        <<<grid, 256, 0, s>>>(pairs, npairs, order, done, counter, status, cost, mv, nsad);
  else
    lowres_search_h264_kernel<uint16_t>
        <<<grid, 256, 0, s>>>(pairs, npairs, order, done, counter, status, cost, mv, nsad);
  return cudaGetLastError();
}

cudaError_t launch_lowres_bi(const LowresDesc& cur, const LowresDesc& r0, const LowresDesc& r1, const rme_mv* m0,
                             const rme_mv* m1, uint32_t* cost, cudaStream_t s) {
  const int grid = (cur.bw * cur.bh + 127) / 128;
  if (!cur.h264)
    lowres_bi_kernel<<<grid, 128, 0, s>>>(cur, r0, r1, m0, m1, cost);
  else if (cur.bytes == 1)
    lowres_bi_h264_kernel<uint8_t><<<grid, 128, 0, s>>>(cur, r0, r1, m0, m1, cost);
  else
    lowres_bi_h264_kernel<uint16_t><<<grid, 128, 0, s>>>(cur, r0, r1, m0, m1, cost);
  return cudaGetLastError();
}

}  // namespace rme
