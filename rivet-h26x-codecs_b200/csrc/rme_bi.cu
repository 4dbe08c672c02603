// HEVC bi-prediction for B units (encode/h265_me.rs): the SATD of a vector
// pair's bi-prediction (satd_bi_at, 4209-4264) and the target block that
// refine_bi (3933-4014) searches one list against, 2 * src minus the other
// list's prediction. One warp per job.
//
// A block is "readable" as the reference's read_at (3630-3655) defines it:
// a whole-sample vector whose block stays within the plane's border, or a
// fractional one whose block stays within HalfPlanes' reach (16 samples, at
// most the border less 4) on a phase HalfPlanes builds (all fifteen up to
// 2,200,000 luma samples, the half phases above; h265_search.rs:35-170).
// Readable blocks are read from the resident planes (the integer plane and
// the fifteen phases, exact uni-predicted samples); any other block is
// interpolated here from the integer plane, its coordinates clamped to the
// picture (the padded plane replicates the edge, so a clamped read is the
// sample the reference's at_clamped window gathers).
#include <cuda_runtime.h>

#include "rme_internal.h"

namespace rme {
namespace {

constexpr unsigned kAll = 0xffffffffu;

// The HEVC luma interpolation taps per quarter fraction
// (hevc/tables_gen.rs:173-191).
__constant__ int8_t c_luma_taps[4][8] = {{0, 0, 0, 0, 0, 0, 0, 0},
                                         {-1, 4, -10, 58, 17, -5, 1, 0},
                                         {-1, 4, -11, 40, 40, -11, 4, -1},
                                         {0, 1, -5, 17, 58, -10, 4, -1}};

template <class S>
__device__ __forceinline__ const S* plane_ptr(const DevPlanes& p, int plane, int x, int y) {
  return (const S*)p.base + (int64_t)plane * p.plane_elems + p.origin + (int64_t)y * p.stride + x;
}

template <class S>
__device__ __forceinline__ int clamped(const DevPlanes& R, int W, int H, int x, int y) {
  return (int)*plane_ptr<S>(R, 0, min(max(x, 0), W - 1), min(max(y, 0), H - 1));
}

// predict14 of one sample (h265_me.rs:4366-4415 through dsp/hevc.rs
// qpel_h / qpel_v / qpel_v2 / copy): the 14-bit prediction at integer
// position (xi, yi) with fractions (fx, fy).
template <class S>
__device__ int pred14(const DevPlanes& R, int W, int H, int bd, int xi, int yi, int fx, int fy) {
  const int shift1 = min(bd, 12) - 8;
  if (fx == 0 && fy == 0) return clamped<S>(R, W, H, xi, yi) << (14 - bd);
  if (fy == 0) {
    int s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += c_luma_taps[fx][k] * clamped<S>(R, W, H, xi - 3 + k, yi);
    return (int)(int16_t)(s >> shift1);
  }
  if (fx == 0) {
    int s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += c_luma_taps[fy][k] * clamped<S>(R, W, H, xi, yi - 3 + k);
    return (int)(int16_t)(s >> shift1);
  }
  int v = 0;
  for (int r = 0; r < 8; ++r) {
    int s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += c_luma_taps[fx][k] * clamped<S>(R, W, H, xi - 3 + k, yi - 3 + r);
    v += c_luma_taps[fy][r] * (int)(int16_t)(s >> shift1);
  }
  return (int)(int16_t)(v >> 6);
}

__device__ __forceinline__ bool readable(const BiDesc& B, int x, int y, int w, int h, int mvx, int mvy) {
  const int xi = x + (mvx >> 2), yi = y + (mvy >> 2);
  if ((mvx & 3) == 0 && (mvy & 3) == 0)
    return xi >= -B.pad && yi >= -B.pad && xi + w <= B.width + B.pad && yi + h <= B.height + B.pad;
  if (!B.quarter && (((mvx | mvy) & 1) != 0)) return false;
  const int ext = min(16, B.pad - 4);
  return xi >= -ext && yi >= -ext && xi + w <= B.width + ext && yi + h <= B.height + ext;
}

// The one-list (uni) prediction sample (row, col) of a block: read where
// the block is readable, else predict14 + uni (dsp/hevc.rs:997-1013).
template <class S>
__device__ __forceinline__ int uni_sample(const BiDesc& B, const DevPlanes& R, bool rd, int x, int y, int mvx, int mvy,
                                          int row, int col) {
  const int xi = x + (mvx >> 2) + col, yi = y + (mvy >> 2) + row, fx = mvx & 3, fy = mvy & 3;
  if (rd) return (int)*plane_ptr<S>(R, fy * 4 + fx, xi, yi);
  const int sh = 14 - B.bd, maxv = (1 << B.bd) - 1;
  return min(max((pred14<S>(R, B.width, B.height, B.bd, xi, yi, fx, fy) + (1 << (sh - 1))) >> sh, 0), maxv);
}

__device__ __forceinline__ uint32_t hadamard4x4_sum(int* d) {
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

// satd_bi_at under default weighting: both blocks readable, the samples
// averaged (a + b + 1) >> 1; otherwise bi of the two 14-bit predictions at
// 15 - bd (dsp/hevc.rs:1015-1031). Lanes take 4x4 tiles in turn.
template <class S>
__global__ void __launch_bounds__(256) bi_satd_kernel(BiDesc B, uint32_t* out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < B.n; i += warps) {
    const rme_bi_job& j = B.jobs[i];
    const int x = j.x, y = j.y, w = j.w, h = j.h;
    const int m0x = j.mv[0].x, m0y = j.mv[0].y, m1x = j.mv[1].x, m1y = j.mv[1].y;
    const DevPlanes& R0 = B.ref[j.ref[0]];
    const DevPlanes& R1 = B.ref[j.ref[1]];
    const bool avg = readable(B, x, y, w, h, m0x, m0y) && readable(B, x, y, w, h, m1x, m1y);
    const int tw = w >> 2, ntiles = tw * (h >> 2);
    const int sh = 15 - B.bd, maxv = (1 << B.bd) - 1;
    uint32_t acc = 0;
    for (int t = lane; t < ntiles; t += 32) {
      const int ty = t / tw, tx = t - ty * tw;
      int d[16];
#pragma unroll 4
      for (int e = 0; e < 16; ++e) {
        const int row = ty * 4 + (e >> 2), col = tx * 4 + (e & 3);
        int pred;
        if (avg) {
          pred = (uni_sample<S>(B, R0, true, x, y, m0x, m0y, row, col) +
                  uni_sample<S>(B, R1, true, x, y, m1x, m1y, row, col) + 1) >> 1;
        } else {
          const int a = pred14<S>(R0, B.width, B.height, B.bd, x + (m0x >> 2) + col, y + (m0y >> 2) + row, m0x & 3,
                                  m0y & 3);
          const int b = pred14<S>(R1, B.width, B.height, B.bd, x + (m1x >> 2) + col, y + (m1y >> 2) + row, m1x & 3,
                                  m1y & 3);
          pred = min(max((a + b + (1 << (sh - 1))) >> sh, 0), maxv);
        }
        d[e] = (int)*plane_ptr<S>(B.src, 0, x + col, y + row) - pred;
      }
      acc += hadamard4x4_sum(d);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kAll, acc, o);
    if (lane == 0) out[i] = acc;
  }
}

// refine_bi's target: clip(2 * src - the other list's prediction), as a
// kBiBlock-wide block per job.
template <class S>
__global__ void __launch_bounds__(256) bi_target_kernel(BiDesc B, S* target) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int maxv = (1 << B.bd) - 1;
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < B.n; i += warps) {
    const rme_bi_job& j = B.jobs[i];
    const int other = 1 - j.list, x = j.x, y = j.y, w = j.w, h = j.h;
    const int mx = j.mv[other].x, my = j.mv[other].y;
    const DevPlanes& R = B.ref[j.ref[other]];
    const bool rd = readable(B, x, y, w, h, mx, my);
    S* dst = target + i * (kBiBlock * kBiBlock);
    for (int e = lane; e < w * h; e += 32) {
      const int row = e / w, col = e - row * w;
      const int p = uni_sample<S>(B, R, rd, x, y, mx, my, row, col);
      const int s = (int)*plane_ptr<S>(B.src, 0, x + col, y + row);
      dst[row * kBiBlock + col] = (S)min(max(2 * s - p, 0), maxv);
    }
  }
}

int grid_of(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, 148 * 16)); }

}  // namespace

cudaError_t launch_bi_satd(const BiDesc& B, uint32_t* satd, cudaStream_t s) {
  if (B.bd == 8)
    bi_satd_kernel<uint8_t><<<grid_of(B.n), 256, 0, s>>>(B, satd);
  else
    bi_satd_kernel<uint16_t><<<grid_of(B.n), 256, 0, s>>>(B, satd);
  return cudaGetLastError();
}

cudaError_t launch_bi_target(const BiDesc& B, void* target, cudaStream_t s) {
  if (B.bd == 8)
    bi_target_kernel<uint8_t><<<grid_of(B.n), 256, 0, s>>>(B, (uint8_t*)target);
  else
    bi_target_kernel<uint16_t><<<grid_of(B.n), 256, 0, s>>>(B, (uint16_t*)target);
  return cudaGetLastError();
}

}  // namespace rme
