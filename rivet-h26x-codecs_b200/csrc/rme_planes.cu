// Per-reference plane builds on the device.
//
// A reference picture is searched by every block of every picture that
// predicts from it, so — as the reference's encoders do on the CPU — its
// sub-sample planes are computed once, when it is uploaded:
//   H.264  build_hpel / hpel_planes (encode/h264_hpel.rs:95-189): the
//          horizontal (b), vertical (h) and centre (j) half-sample planes.
//   HEVC   HalfPlanes::new (encode/h265_search.rs:79-170): the fifteen
//          fractional phases, each the exact uni-predicted sample of
//          8.5.3.3.3.1 (8-tap, shift1 = Min(4, BitDepth-8), second pass
//          >> 6, (x + offset) >> (14 - BitDepth) and clip).
// The reference's planes hold a copy of the integer sample where a filter
// window would leave the padded plane, and HalfPlanes stops REACH samples
// outside the picture; neither region is ever read by a search whose
// window rules hold (search_bounds, clamp_pos), so here every position is
// computed over the edge-replicated plane, which gives the reference's
// value wherever the reference computes one.
#include <cuda_runtime.h>

#include "rme_internal.h"

namespace rme {
namespace {

template <class S>
__global__ void pad_plane_kernel(const S* __restrict__ src, int w, int h, int sstride, S* __restrict__ dst,
                                 int dstride, int prow, int pcol, int pad) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= pcol || y >= prow) return;
  // In place (src is the plane's own visible picture): only the border is
  // written, and it reads only the visible picture.
  if (src == dst + (int64_t)pad * dstride + pad && x >= pad && x < pad + w && y >= pad && y < pad + h) return;
  int sx = min(max(x - pad, 0), w - 1);
  int sy = min(max(y - pad, 0), h - 1);
  dst[(int64_t)y * dstride + x] = src[(int64_t)sy * sstride + sx];
}

__device__ __forceinline__ int tap6(int a, int b, int c, int d, int e, int f) {
  return a + f - 5 * (b + e) + 20 * (c + d);
}

// b, h, j of every padded position (x, y): reads of G clamped to the padded
// plane, i.e. of the edge-replicated picture.
template <class S>
__global__ void h264_hpel_kernel(const S* __restrict__ g, S* __restrict__ pb, S* __restrict__ ph, S* __restrict__ pj,
                                 int stride, int prow, int pcol, int maxv) {
  constexpr int TX = 32, TY = 8;
  __shared__ int tile[TY + 5][TX + 5];  // G over rows y-2..y+TY+2, cols x-2..x+TX+2
  __shared__ int vin[TY][TX + 5];       // vertical six-tap, unclipped
  int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  int tid = threadIdx.y * TX + threadIdx.x;
  for (int i = tid; i < (TY + 5) * (TX + 5); i += TX * TY) {
    int ty = i / (TX + 5), tx = i % (TX + 5);
    int gx = min(max(x0 + tx - 2, 0), pcol - 1), gy = min(max(y0 + ty - 2, 0), prow - 1);
    tile[ty][tx] = g[(int64_t)gy * stride + gx];
  }
  __syncthreads();
  for (int i = tid; i < TY * (TX + 5); i += TX * TY) {
    int ty = i / (TX + 5), tx = i % (TX + 5);
    vin[ty][tx] = tap6(tile[ty][tx], tile[ty + 1][tx], tile[ty + 2][tx], tile[ty + 3][tx], tile[ty + 4][tx],
                       tile[ty + 5][tx]);
  }
  __syncthreads();
  int tx = threadIdx.x, ty = threadIdx.y, x = x0 + tx, y = y0 + ty;
  if (x >= pcol || y >= prow) return;
  const int* r = &tile[ty + 2][tx];
  int b = tap6(r[0], r[1], r[2], r[3], r[4], r[5]);
  int v = vin[ty][tx + 2];
  const int* q = &vin[ty][tx];
  int j = tap6(q[0], q[1], q[2], q[3], q[4], q[5]);
  int64_t o = (int64_t)y * stride + x;
  pb[o] = (S)min(max((b + 16) >> 5, 0), maxv);
  ph[o] = (S)min(max((v + 16) >> 5, 0), maxv);
  pj[o] = (S)min(max((j + 512) >> 10, 0), maxv);
}

__constant__ int8_t c_qpel[4][8] = {{0, 0, 0, 0, 0, 0, 0, 0},
                                    {-1, 4, -10, 58, 17, -5, 1, 0},
                                    {-1, 4, -11, 40, 40, -11, 4, -1},
                                    {0, 1, -5, 17, 58, -10, 4, -1}};

// The fifteen phases of every padded position: the horizontal pass of each
// fraction over TY + 7 rows kept in shared memory (int16, as the
// reference's intermediate), the vertical passes from it. A tile of 32 x 8
// positions, blocks of 32 x 4 threads (two rows each): one block fits in
// the registers the resident engine leaves free on every SM, so a
// picture's planes are built while the engine runs.
constexpr int kPhaseTX = 32, kPhaseTY = 8, kPhaseRows = 4;
template <class S>
__global__ void hevc_phase_kernel(const S* g, S* planes, int64_t plane_elems, int stride,
                                  int prow, int pcol, int bd) {
  constexpr int TX = kPhaseTX, TY = kPhaseTY, NT = kPhaseTX * kPhaseRows;
  __shared__ int tile[TY + 7][TX + 7];
  __shared__ int16_t hp[3][TY + 7][TX];
  int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  int tid = threadIdx.y * TX + threadIdx.x;
  int shift1 = min(bd, 12) - 8, shift3 = 14 - bd, maxv = (1 << bd) - 1, round3 = 1 << (shift3 - 1);
  for (int i = tid; i < (TY + 7) * (TX + 7); i += NT) {
    int ty = i / (TX + 7), tx = i % (TX + 7);
    int gx = min(max(x0 + tx - 3, 0), pcol - 1), gy = min(max(y0 + ty - 3, 0), prow - 1);
    tile[ty][tx] = g[(int64_t)gy * stride + gx];
  }
  __syncthreads();
  for (int i = tid; i < 3 * (TY + 7) * TX; i += NT) {
    int f = i / ((TY + 7) * TX), rem = i % ((TY + 7) * TX), ty = rem / TX, tx = rem % TX;
    int acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += c_qpel[f + 1][k] * tile[ty][tx + k];
    hp[f][ty][tx] = (int16_t)(acc >> shift1);
  }
  __syncthreads();
  const int tx = threadIdx.x, x = x0 + tx;
  for (int ty = threadIdx.y; ty < TY; ty += kPhaseRows) {
    const int y = y0 + ty;
    if (x >= pcol || y >= prow) return;
    const int64_t o = (int64_t)y * stride + x;
    auto put = [&](int phase, int v14) {
      int v = min(max(((int)(int16_t)v14 + round3) >> shift3, 0), maxv);
      planes[(int64_t)phase * plane_elems + o] = (S)v;
    };
    for (int fx = 1; fx < 4; ++fx) put(fx, hp[fx - 1][ty + 3][tx]);
    for (int fy = 1; fy < 4; ++fy) {
      int acc = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) acc += c_qpel[fy][k] * tile[ty + k][tx + 3];
      put(fy * 4, acc >> shift1);
      for (int fx = 1; fx < 4; ++fx) {
        int a2 = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) a2 += c_qpel[fy][k] * (int)hp[fx - 1][ty + k][tx];
        put(fy * 4 + fx, a2 >> 6);
      }
    }
  }
}

}  // namespace

cudaError_t launch_pad_plane(const void* src, int bd, int w, int h, int sstride, DevPlanes dst, int cw, int ch,
                             int pad, cudaStream_t s) {
  int prow = ch + 2 * pad, pcol = cw + 2 * pad;
  dim3 blk(32, 8), grd((pcol + 31) / 32, (prow + 7) / 8);
  prefer_max_shared(pad_plane_kernel<uint8_t>);
  prefer_max_shared(pad_plane_kernel<uint16_t>);
  if (bd == 8)
    pad_plane_kernel<uint8_t><<<grd, blk, 0, s>>>((const uint8_t*)src, w, h, sstride, (uint8_t*)dst.base, dst.stride,
                                                  prow, pcol, pad);
  else
    pad_plane_kernel<uint16_t><<<grd, blk, 0, s>>>((const uint16_t*)src, w, h, sstride, (uint16_t*)dst.base,
                                                   dst.stride, prow, pcol, pad);
  return cudaGetLastError();
}

cudaError_t launch_h264_hpel(DevPlanes p, int bd, int cw, int ch, int pad, cudaStream_t s) {
  int prow = ch + 2 * pad, pcol = cw + 2 * pad;
  dim3 blk(32, 8), grd((pcol + 31) / 32, (prow + 7) / 8);
  prefer_max_shared(h264_hpel_kernel<uint8_t>);
  prefer_max_shared(h264_hpel_kernel<uint16_t>);
  if (bd == 8) {
    auto b = (uint8_t*)p.base;
    h264_hpel_kernel<uint8_t><<<grd, blk, 0, s>>>(b, b + p.plane_elems, b + 2 * p.plane_elems, b + 3 * p.plane_elems,
                                                  p.stride, prow, pcol, 255);
  } else {
    auto b = (uint16_t*)p.base;
    h264_hpel_kernel<uint16_t><<<grd, blk, 0, s>>>(b, b + p.plane_elems, b + 2 * p.plane_elems,
                                                   b + 3 * p.plane_elems, p.stride, prow, pcol, (1 << bd) - 1);
  }
  return cudaGetLastError();
}

cudaError_t launch_hevc_phases(DevPlanes p, int bd, int w, int h, int pad, cudaStream_t s) {
  int prow = h + 2 * pad, pcol = w + 2 * pad;
  dim3 blk(kPhaseTX, kPhaseRows), grd((pcol + kPhaseTX - 1) / kPhaseTX, (prow + kPhaseTY - 1) / kPhaseTY);
  prefer_max_shared(hevc_phase_kernel<uint8_t>);
  prefer_max_shared(hevc_phase_kernel<uint16_t>);
  if (bd == 8)
    hevc_phase_kernel<uint8_t><<<grd, blk, 0, s>>>((const uint8_t*)p.base, (uint8_t*)p.base, p.plane_elems, p.stride,
                                                   prow, pcol, bd);
  else
    hevc_phase_kernel<uint16_t><<<grd, blk, 0, s>>>((const uint16_t*)p.base, (uint16_t*)p.base, p.plane_elems,
                                                    p.stride, prow, pcol, bd);
  return cudaGetLastError();
}

}  // namespace rme
