// Weighted prediction for the search (explicit weights): the weighted copy
// of a reference plane the motion search scores against (H.264
// weighted_search_plane, encode/h264_me.rs:653-672; HEVC
// weighted_search_plane, encode/h265_me.rs:4275-4293), and the two passes
// the encoders' weight fit makes over a picture pair (wp_moments and
// weighted_sad, dsp/distortion.rs:206-252).
//
// All three read or write every sample once: they are HBM-bound streams
// (the plane as 16-byte vectors; the picture pair row by row with a
// block-wide reduction into 64-bit sums).
#include <cuda_runtime.h>

#include "rme_internal.h"

namespace rme {
namespace {

constexpr unsigned kAll = 0xffffffffu;

struct WeightArgs {
  int codec, bd, log_wd, weight, offset;
};

__device__ __forceinline__ int weighted_sample(const WeightArgs& a, int v) {
  const int maxv = (1 << a.bd) - 1;
  int p;
  if (a.codec == RME_CODEC_H264) {
    const int x = v * a.weight;
    p = a.log_wd >= 1 ? ((x + (1 << (a.log_wd - 1))) >> a.log_wd) + a.offset : x + a.offset;
  } else {
    p = (((v << (14 - a.bd)) * a.weight + (1 << (a.log_wd - 1))) >> a.log_wd) + a.offset;
  }
  return min(max(p, 0), maxv);
}

// Every sample of the padded plane, border included (the weighting is per
// sample, so it commutes with the border's replication): 16 bytes per
// thread per step.
template <class S>
__global__ void weighted_plane_kernel(const uint4* __restrict__ src, uint4* __restrict__ dst, int64_t nvec,
                                      WeightArgs a) {
  constexpr int N = 16 / sizeof(S);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += (int64_t)gridDim.x * blockDim.x) {
    uint4 v = src[i];
    S* e = reinterpret_cast<S*>(&v);
#pragma unroll
    for (int k = 0; k < N; ++k) e[k] = (S)weighted_sample(a, (int)e[k]);
    dst[i] = v;
  }
}

template <class T>
__device__ __forceinline__ T block_sum(T v, T* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kAll, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T t = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) t += red[i];
  return t;
}

// wp_moments: sums of r, c, r*r, r*c, |c - r| over the display area, each
// block a band of rows, one 64-bit atomic per sum per block.
template <class S>
__global__ void __launch_bounds__(256) wp_moments_kernel(const S* cur, int cs, const S* ref, int rs, int w, int h,
                                                         unsigned long long* out) {
  __shared__ unsigned long long red[8];
  unsigned long long sr = 0, sc = 0, srr = 0, src = 0, sad = 0;
  for (int y = blockIdx.x; y < h; y += gridDim.x) {
    const S* cr = cur + (int64_t)y * cs;
    const S* rr = ref + (int64_t)y * rs;
    uint32_t a = 0, b = 0, d = 0;  // a row's sums fit 32 bits (w * 4095 * 2)
    unsigned long long aa = 0, ab = 0;
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
      const uint32_t r = rr[x], c = cr[x];
      a += r;
      b += c;
      aa += r * r;
      ab += r * c;
      d += r > c ? r - c : c - r;
    }
    sr += a;
    sc += b;
    srr += aa;
    src += ab;
    sad += d;
  }
  unsigned long long v[5] = {sr, sc, srr, src, sad};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const unsigned long long t = block_sum(v[k], red);
    if (threadIdx.x == 0 && t) atomicAdd(out + k, t);
  }
}

// weighted_sad: sum of |clip(((r * weight + round) >> shift) + offset) - c|.
template <class S>
__global__ void __launch_bounds__(256) weighted_sad_kernel(const S* cur, int cs, const S* ref, int rs, int w, int h,
                                                           int weight, int shift, int offset, int maxv,
                                                           unsigned long long* out) {
  __shared__ unsigned long long red[8];
  const int round = shift >= 1 ? 1 << (shift - 1) : 0;
  unsigned long long sad = 0;
  for (int y = blockIdx.x; y < h; y += gridDim.x) {
    const S* cr = cur + (int64_t)y * cs;
    const S* rr = ref + (int64_t)y * rs;
    uint32_t d = 0;
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
      const int p = min(max((((int)rr[x] * weight + round) >> shift) + offset, 0), maxv);
      d += (uint32_t)abs(p - (int)cr[x]);
    }
    sad += d;
  }
  const unsigned long long t = block_sum(sad, red);
  if (threadIdx.x == 0 && t) atomicAdd(out, t);
}

int rows_grid(int h) { return std::max(1, std::min(h, 148 * 4)); }

}  // namespace

cudaError_t launch_weighted_plane(const void* src, void* dst, int64_t bytes, int codec, int bd, int log_wd, int weight,
                                  int offset, cudaStream_t s) {
  const WeightArgs a{codec, bd, log_wd, weight, offset};
  const int64_t nvec = bytes / 16;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nvec + 255) / 256, 148 * 8));
  if (bd == 8)
    weighted_plane_kernel<uint8_t><<<grid, 256, 0, s>>>((const uint4*)src, (uint4*)dst, nvec, a);
  else
    weighted_plane_kernel<uint16_t><<<grid, 256, 0, s>>>((const uint4*)src, (uint4*)dst, nvec, a);
  return cudaGetLastError();
}

cudaError_t launch_wp_moments(const void* cur, const void* ref, int stride, int bd, int w, int h,
                              unsigned long long* out, cudaStream_t s) {
  if (bd == 8)
    wp_moments_kernel<uint8_t><<<rows_grid(h), 256, 0, s>>>((const uint8_t*)cur, stride, (const uint8_t*)ref, stride,
                                                            w, h, out);
  else
    wp_moments_kernel<uint16_t><<<rows_grid(h), 256, 0, s>>>((const uint16_t*)cur, stride, (const uint16_t*)ref,
                                                             stride, w, h, out);
  return cudaGetLastError();
}

cudaError_t launch_weighted_sad(const void* cur, const void* ref, int stride, int bd, int w, int h, int weight,
                                int shift, int offset, unsigned long long* out, cudaStream_t s) {
  const int maxv = (1 << bd) - 1;
  if (bd == 8)
    weighted_sad_kernel<uint8_t><<<rows_grid(h), 256, 0, s>>>((const uint8_t*)cur, stride, (const uint8_t*)ref,
                                                              stride, w, h, weight, shift, offset, maxv, out);
  else
    weighted_sad_kernel<uint16_t><<<rows_grid(h), 256, 0, s>>>((const uint16_t*)cur, stride, (const uint16_t*)ref,
                                                               stride, w, h, weight, shift, offset, maxv, out);
  return cudaGetLastError();
}

}  // namespace rme
