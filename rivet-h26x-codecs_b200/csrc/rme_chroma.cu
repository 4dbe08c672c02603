// Chroma prediction of chosen vectors and the batched distortion kernels.
//
// Chroma (4:2:0): a luma vector in quarter samples is the chroma vector in
// eighth samples. HEVC is predict_block's chroma arm (hevc/inter.rs:555-660):
// the 4-tap EPEL filter (hevc/tables_gen.rs:173-191) horizontally and/or
// vertically at 14-bit precision (dsp/hevc.rs:757-821; h then v2 on the int16
// intermediate when both fractions are non-zero), then uni rounding
// (dsp/hevc.rs:997-1013). H.264 is chroma_pred_into (h264_me.rs:812-837):
// the bilinear weights (8-xf)(8-yf), xf(8-yf), (8-xf)yf, xf*yf and
// (v + 32) >> 6 (dsp/h264.rs:499-520). Every reference read, inside the
// reference's padding or outside it, is the edge-replicated picture, so the
// kernel reads the unpadded planes with clamped coordinates.
//
// Distortion batches: dsp/distortion.rs SadFn / SatdFn applied to n pairs
// of blocks, one warp per pair.
#include <cuda_runtime.h>

#include "rme_internal.h"

namespace rme {
namespace {

__constant__ int8_t c_epel[8][4] = {{0, 0, 0, 0},     {-2, 58, 10, -2}, {-4, 54, 16, -2}, {-6, 46, 28, -4},
                                    {-4, 36, 36, -4}, {-4, 28, 46, -6}, {-2, 16, 54, -4}, {-2, 10, 58, -2}};

template <class S>
__device__ __forceinline__ int at_clamped(const S* p, int cw, int ch, int x, int y) {
  return (int)p[(size_t)min(max(y, 0), ch - 1) * cw + min(max(x, 0), cw - 1)];
}

// One block per CTA; its threads cover the block's Cb then Cr samples.
template <class S>
__global__ void chroma_kernel(const S* __restrict__ cb, const S* __restrict__ cr, int bd, int codec, int cw, int ch,
                              const int32_t* __restrict__ blocks, const rme_mv* __restrict__ mvs,
                              const int64_t* __restrict__ out_off, S* __restrict__ out) {
  const int i = blockIdx.x;
  const int x = blocks[4 * i] / 2, y = blocks[4 * i + 1] / 2, w = blocks[4 * i + 2] / 2, h = blocks[4 * i + 3] / 2;
  const int mx = mvs[i].x, my = mvs[i].y;
  const int xi = x + (mx >> 3), yi = y + (my >> 3), xf = mx & 7, yf = my & 7;
  S* o = out + out_off[i];
  const int shift1 = min(bd, 12) - 8, shift3 = 14 - bd, maxv = (1 << bd) - 1;
  const int round3 = shift3 > 0 ? 1 << (shift3 - 1) : 0;
  for (int k = threadIdx.x; k < 2 * w * h; k += blockDim.x) {
    const int c = k >= w * h, j = k - c * w * h, yy = j / w, xx = j - yy * w;
    const S* pl = c ? cr : cb;
    const int px = xi + xx, py = yi + yy;
    int v;
    if (codec == RME_CODEC_HEVC) {
      int v14;
      if (xf == 0 && yf == 0) {
        v14 = at_clamped(pl, cw, ch, px, py) << shift3;
      } else if (yf == 0) {
        int acc = 0;
#pragma unroll
        for (int t = 0; t < 4; ++t) acc += c_epel[xf][t] * at_clamped(pl, cw, ch, px - 1 + t, py);
        v14 = (int16_t)(acc >> shift1);
      } else if (xf == 0) {
        int acc = 0;
#pragma unroll
        for (int t = 0; t < 4; ++t) acc += c_epel[yf][t] * at_clamped(pl, cw, ch, px, py - 1 + t);
        v14 = (int16_t)(acc >> shift1);
      } else {
        int acc2 = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          int acc = 0;
#pragma unroll
          for (int t = 0; t < 4; ++t) acc += c_epel[xf][t] * at_clamped(pl, cw, ch, px - 1 + t, py - 1 + u);
          acc2 += c_epel[yf][u] * (int)(int16_t)(acc >> shift1);
        }
        v14 = (int16_t)(acc2 >> 6);
      }
      v = min(max((v14 + round3) >> shift3, 0), maxv);
    } else {
      const int A = (8 - xf) * (8 - yf), B = xf * (8 - yf), C = (8 - xf) * yf, D = xf * yf;
      v = (A * at_clamped(pl, cw, ch, px, py) + B * at_clamped(pl, cw, ch, px + 1, py) +
           C * at_clamped(pl, cw, ch, px, py + 1) + D * at_clamped(pl, cw, ch, px + 1, py + 1) + 32) >> 6;
    }
    o[k] = (S)v;
  }
}

// dsp/distortion.rs:326-381, one 4x4 tile of differences.
__device__ __forceinline__ uint32_t tile_satd(int d[16]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int a = d[i * 4], b = d[i * 4 + 1], c = d[i * 4 + 2], e = d[i * 4 + 3];
    int s0 = a + e, s1 = b + c, s2 = b - c, s3 = a - e;
    d[i * 4] = s0 + s1;
    d[i * 4 + 1] = s3 + s2;
    d[i * 4 + 2] = s0 - s1;
    d[i * 4 + 3] = s3 - s2;
  }
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int a = d[j], b = d[4 + j], c = d[8 + j], e = d[12 + j];
    int s0 = a + e, s1 = b + c, s2 = b - c, s3 = a - e;
    sum += abs(s0 + s1) + abs(s3 + s2) + abs(s0 - s1) + abs(s3 - s2);
  }
  return (sum + 1) >> 1;
}

// One warp per pair: SAD over samples (lanes stride the block), SATD over
// 4x4 tiles (lanes stride the tiles); the warp's sum to out[i].
template <class S>
__global__ void dist_batch_kernel(bool satd, const S* __restrict__ a, int64_t as, const int64_t* __restrict__ aoff,
                                  const S* __restrict__ b, int64_t bs, const int64_t* __restrict__ boff, int w, int h,
                                  int n, uint32_t* __restrict__ out) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= n) return;
  const S* pa = a + aoff[i];
  const S* pb = b + boff[i];
  uint32_t acc = 0;
  if (!satd) {
    for (int k = lane; k < w * h; k += 32) {
      const int y = k / w, x = k - y * w;
      acc += (uint32_t)abs((int)pa[y * as + x] - (int)pb[y * bs + x]);
    }
  } else {
    const int tw = w >> 2, nt = tw * (h >> 2);
    for (int t = lane; t < nt; t += 32) {
      const int ty = t / tw, tx = t - ty * tw;
      int d[16];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
          d[r * 4 + c] = (int)pa[(ty * 4 + r) * as + tx * 4 + c] - (int)pb[(ty * 4 + r) * bs + tx * 4 + c];
      acc += tile_satd(d);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[i] = acc;
}

}  // namespace

cudaError_t launch_chroma(const void* cb, const void* cr, int bd, int codec, int cw, int ch, int cstride,
                          int nblocks, const int32_t* blocks, const rme_mv* mvs, const int64_t* out_off, void* out,
                          cudaStream_t s) {
  (void)cstride;  // the planes are stored packed, cw samples per row
  if (nblocks <= 0) return cudaSuccess;
  if (bd == 8)
    chroma_kernel<uint8_t><<<nblocks, 128, 0, s>>>((const uint8_t*)cb, (const uint8_t*)cr, bd, codec, cw, ch, blocks,
                                                   mvs, out_off, (uint8_t*)out);
  else
    chroma_kernel<uint16_t><<<nblocks, 128, 0, s>>>((const uint16_t*)cb, (const uint16_t*)cr, bd, codec, cw, ch,
                                                    blocks, mvs, out_off, (uint16_t*)out);
  return cudaGetLastError();
}

cudaError_t launch_dist_batch(bool satd, const void* a, int64_t as, const int64_t* aoff, const void* b, int64_t bs,
                              const int64_t* boff, int w, int h, int bd, int n, uint32_t* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int warps = 8, grid = (n + warps - 1) / warps;
  if (bd == 8)
    dist_batch_kernel<uint8_t><<<grid, warps * 32, 0, s>>>(satd, (const uint8_t*)a, as, aoff, (const uint8_t*)b, bs,
                                                            boff, w, h, n, out);
  else
    dist_batch_kernel<uint16_t><<<grid, warps * 32, 0, s>>>(satd, (const uint16_t*)a, as, aoff, (const uint16_t*)b,
                                                             bs, boff, w, h, n, out);
  return cudaGetLastError();
}

}  // namespace rme
