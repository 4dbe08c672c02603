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

// satd_bi_at: under default weighting with both blocks readable, the
// samples averaged (a + b + 1) >> 1; otherwise bi of the two 14-bit
// predictions at 15 - bd (dsp/hevc.rs:1015-1031), or under explicit
// weighting weighted_bi of them (dsp/hevc.rs:1064-1086). Lanes take 4x4
// tiles in turn.
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
    const bool avg = !B.wp && readable(B, x, y, w, h, m0x, m0y) && readable(B, x, y, w, h, m1x, m1y);
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
          pred = B.wp ? (a * B.w0 + b * B.w1 + ((B.o0 + B.o1 + 1) << B.log2_wd)) >> (B.log2_wd + 1)
                      : (a + b + (1 << (sh - 1))) >> sh;
          pred = min(max(pred, 0), maxv);
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

// ---- H.264 B macroblocks: bi_refine (h264_analyse.rs:2793-2900) -------------

// The quarter-sample positions' plane views (h264_hpel.rs QPEL, 205-281):
// per position, plane and offset of one view, then of the second view
// averaged with it (plane -1: one view only). Planes: G, b, h, j.
__constant__ int8_t c_qpel_views[16][6] = {
    {0, 0, 0, -1, 0, 0}, {0, 0, 0, 1, 0, 0}, {1, 0, 0, -1, 0, 0}, {1, 0, 0, 0, 1, 0},
    {0, 0, 0, 2, 0, 0},  {1, 0, 0, 2, 0, 0}, {1, 0, 0, 3, 0, 0},  {1, 0, 0, 2, 1, 0},
    {2, 0, 0, -1, 0, 0}, {2, 0, 0, 3, 0, 0}, {3, 0, 0, -1, 0, 0}, {3, 0, 0, 2, 1, 0},
    {2, 0, 0, 0, 0, 1},  {2, 0, 0, 1, 0, 1}, {3, 0, 0, 1, 0, 1},  {2, 1, 0, 1, 0, 1},
};
__constant__ int8_t c_bi_ring[8][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};

// MeRef::pred's sample (row, col) of a block at (x, y) and vector (mx, my).
template <class S>
__device__ __forceinline__ int qpel_sample(const DevPlanes& R, int x, int y, int mx, int my, int row, int col) {
  const int8_t* q = c_qpel_views[(my & 3) * 4 + (mx & 3)];
  const int xi = x + (mx >> 2) + col, yi = y + (my >> 2) + row;
  const int a = *plane_ptr<S>(R, q[0], xi + q[1], yi + q[2]);
  if (q[3] < 0) return a;
  return (a + (int)*plane_ptr<S>(R, q[3], xi + q[4], yi + q[5]) + 1) >> 1;
}

struct H264BiDesc {
  DevPlanes src;
  DevPlanes ref[RME_MAX_REFS];
  const uint16_t* tab;  // MvCostTable
  const rme_h264_bi_job* jobs;
  int32_t n, rounds, npts;
  rme_mv* mv_out;
  uint32_t* cost_out;
};

__device__ __forceinline__ uint32_t bi_rate(const uint16_t* tab, int m0x, int m0y, int m1x, int m1y,
                                            const rme_h264_bi_job& j) {
  auto comp = [&](int d) { return (uint32_t)__ldg(&tab[min(max(d, -kMvSpan), kMvSpan) + kMvSpan]); };
  return comp(m0x - j.mvp[0].x) + comp(m0y - j.mvp[0].y) + comp(m1x - j.mvp[1].x) + comp(m1y - j.mvp[1].y);
}

// One warp per pair. A scoring pass gives each of 8 groups of 4 lanes one
// candidate pair; a lane takes the group's 4x4 tiles sub, sub + 4, ...
template <class S>
__global__ void __launch_bounds__(256) h264_bi_kernel(H264BiDesc B) {
  const int lane = threadIdx.x & 31, g = lane >> 2, sub = lane & 3;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < B.n; i += warps) {
    const rme_h264_bi_job& j = B.jobs[i];
    const int x = j.x, y = j.y, w = j.w, h = j.h, tw = w >> 2, ntiles = tw * (h >> 2);
    const DevPlanes& R0 = B.ref[j.ref[0]];
    const DevPlanes& R1 = B.ref[j.ref[1]];
    // The SATD of group g's pair (ok), summed over its four lanes.
    auto score = [&](bool ok, int m0x, int m0y, int m1x, int m1y) -> uint32_t {
      uint32_t acc = 0;
      if (ok)
        for (int t = sub; t < ntiles; t += 4) {
          const int ty = t / tw, tx = t - ty * tw;
          int d[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int row = ty * 4 + (e >> 2), col = tx * 4 + (e & 3);
            const int pr = (qpel_sample<S>(R0, x, y, m0x, m0y, row, col) +
                            qpel_sample<S>(R1, x, y, m1x, m1y, row, col) + 1) >> 1;
            d[e] = (int)*plane_ptr<S>(B.src, 0, x + col, y + row) - pr;
          }
          acc += hadamard4x4_sum(d);
        }
      acc += __shfl_xor_sync(kAll, acc, 1);
      acc += __shfl_xor_sync(kAll, acc, 2);
      return acc;
    };
    int bx[2] = {j.mv[0].x, j.mv[1].x}, by[2] = {j.mv[0].y, j.mv[1].y};
    uint32_t cost = __shfl_sync(kAll, score(g == 0, bx[0], by[0], bx[1], by[1]), 0) +
                    bi_rate(B.tab, bx[0], by[0], bx[1], by[1], j);
    const int nr = cost > j.limit ? 0 : B.rounds;
    for (int it = 0; it < nr; ++it) {
      const int b0x = bx[0], b0y = by[0], b1x = bx[1], b1y = by[1];
      for (int l = 0; l < 2; ++l) {
        const int cx = bx[l], cy = by[l];
        int mx[2] = {bx[0], bx[1]}, my[2] = {by[0], by[1]};
        mx[l] = cx + c_bi_ring[g][0];
        my[l] = cy + c_bi_ring[g][1];
        const uint32_t sc = score(g < B.npts, mx[0], my[0], mx[1], my[1]);
        // In order, as the reference takes them (all lanes alike).
        for (int k = 0; k < B.npts; ++k) {
          const uint32_t s = __shfl_sync(kAll, sc, 4 * k);
          // The ring is around the list's vector at the ring's start; the
          // held list's vector does not change within the ring.
          int kx[2] = {bx[0], bx[1]}, ky[2] = {by[0], by[1]};
          kx[l] = cx + c_bi_ring[k][0];
          ky[l] = cy + c_bi_ring[k][1];
          const uint32_t rc = bi_rate(B.tab, kx[0], ky[0], kx[1], ky[1], j);
          if (rc >= cost) continue;
          if (s + rc < cost) {
            cost = s + rc;
            bx[0] = kx[0];
            by[0] = ky[0];
            bx[1] = kx[1];
            by[1] = ky[1];
          }
        }
      }
      if (bx[0] == b0x && by[0] == b0y && bx[1] == b1x && by[1] == b1y) break;
    }
    if (lane == 0) {
      B.mv_out[2 * i].x = (int16_t)bx[0];
      B.mv_out[2 * i].y = (int16_t)by[0];
      B.mv_out[2 * i + 1].x = (int16_t)bx[1];
      B.mv_out[2 * i + 1].y = (int16_t)by[1];
      B.cost_out[i] = cost;
    }
  }
}

// ---- HEVC weighted lists: refine_subpel under explicit weighting -------------

// mv_bits and the rate (h265_search.rs:212-255, h265_me.rs:3890).
__device__ __forceinline__ uint32_t wr_cbits(int d) {
  const uint32_t a = (uint32_t)abs(d);
  return a == 0 ? 1u : 3u + 2u * (31u - __clz(a));
}
__device__ __forceinline__ uint32_t wr_rate(float lam, int mx, int my, const rme_job& j) {
  const uint32_t b0 = wr_cbits(mx - j.mvp[0].x) + wr_cbits(my - j.mvp[0].y);
  const uint32_t b1 = wr_cbits(mx - j.mvp[1].x) + wr_cbits(my - j.mvp[1].y);
  return __float2uint_rz(__fmul_rn(lam, __uint2float_rn(min(b0, b1) + 1u)));
}

struct WeightedRefine {
  BiDesc B;                 // source, references, sizes
  const rme_job* jobs;      // start = seeds[0], AMVP pair mvp
  int32_t log2_wd, weight, offset, quarter_cross;
  float lam;
  rme_result* out;
};

// One warp per job: refine_subpel (h265_me.rs:3868-3922) with every
// candidate scored by satd_at_weighted's explicit arm (4057-4073): the
// 14-bit prediction (interpolated here from the integer plane), then
// weighted_uni (dsp/hevc.rs:1036-1062), then SATD. Lanes take 4x4 tiles.
template <class S>
__global__ void __launch_bounds__(256) weighted_refine_kernel(WeightedRefine P) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const BiDesc& B = P.B;
  const int maxv = (1 << B.bd) - 1;
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < B.n; i += warps) {
    const rme_job& j = P.jobs[i];
    const int x = j.x, y = j.y, w = j.w, h = j.h, tw = w >> 2, ntiles = tw * (h >> 2);
    const DevPlanes& R = B.ref[j.ref];
    auto satd_w = [&](int mx, int my) -> uint32_t {
      uint32_t acc = 0;
      for (int t = lane; t < ntiles; t += 32) {
        const int ty = t / tw, tx = t - ty * tw;
        int d[16];
#pragma unroll 4
        for (int e = 0; e < 16; ++e) {
          const int row = ty * 4 + (e >> 2), col = tx * 4 + (e & 3);
          const int p14 =
              pred14<S>(R, B.width, B.height, B.bd, x + (mx >> 2) + col, y + (my >> 2) + row, mx & 3, my & 3);
          const int v = P.log2_wd >= 1 ? ((p14 * P.weight + (1 << (P.log2_wd - 1))) >> P.log2_wd) + P.offset
                                       : p14 * P.weight + P.offset;
          d[e] = (int)*plane_ptr<S>(B.src, 0, x + col, y + row) - min(max(v, 0), maxv);
        }
        acc += hadamard4x4_sum(d);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kAll, acc, o);
      return acc;
    };
    const int sx = j.seeds[0].x, sy = j.seeds[0].y;
    int bx = sx, by = sy;
    uint32_t bsatd = satd_w(bx, by), bcost = bsatd + wr_rate(P.lam, bx, by, j), nsatd = 1;
    for (int step = 2; step >= 1; --step) {
      const int cx = bx, cy = by;
      const bool cross = step == 1 && P.quarter_cross != 0;
      for (int qy = -1; qy <= 1; ++qy)
        for (int qx = -1; qx <= 1; ++qx) {
          if ((qx == 0 && qy == 0) || (cross && qx != 0 && qy != 0)) continue;
          const int mx = (int)(int16_t)(cx + qx * step), my = (int)(int16_t)(cy + qy * step);
          const uint32_t sat = satd_w(mx, my), c = sat + wr_rate(P.lam, mx, my, j);
          ++nsatd;
          if (c < bcost) {
            bcost = c;
            bsatd = sat;
            bx = mx;
            by = my;
          }
        }
    }
    if (lane == 0) {
      rme_result r;
      r.mv.x = (int16_t)bx;
      r.mv.y = (int16_t)by;
      r.ref = j.ref;
      r.cost = bcost;
      r.satd = bsatd;
      r.int_mv.x = (int16_t)sx;
      r.int_mv.y = (int16_t)sy;
      r.int_cost = 0;
      r.n_sad = 0;
      r.n_satd = nsatd;
      P.out[i] = r;
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

cudaError_t launch_h264_bi(const DevPlanes& src, const DevPlanes* refs, int nref, int bd, const uint16_t* tab,
                           const rme_h264_bi_job* jobs, int n, int rounds, int npts, rme_mv* mv_out,
                           uint32_t* cost_out, cudaStream_t s) {
  H264BiDesc B{};
  B.src = src;
  for (int r = 0; r < nref; ++r) B.ref[r] = refs[r];
  B.tab = tab;
  B.jobs = jobs;
  B.n = n;
  B.rounds = rounds;
  B.npts = npts;
  B.mv_out = mv_out;
  B.cost_out = cost_out;
  if (bd == 8)
    h264_bi_kernel<uint8_t><<<grid_of(n), 256, 0, s>>>(B);
  else
    h264_bi_kernel<uint16_t><<<grid_of(n), 256, 0, s>>>(B);
  return cudaGetLastError();
}

cudaError_t launch_weighted_refine(const BiDesc& B, const rme_job* jobs, int log2_wd, int weight, int offset,
                                   int quarter_cross, float lam, rme_result* out, cudaStream_t s) {
  WeightedRefine P{};
  P.B = B;
  P.jobs = jobs;
  P.log2_wd = log2_wd;
  P.weight = weight;
  P.offset = offset;
  P.quarter_cross = quarter_cross;
  P.lam = lam;
  P.out = out;
  if (B.bd == 8)
    weighted_refine_kernel<uint8_t><<<grid_of(B.n), 256, 0, s>>>(P);
  else
    weighted_refine_kernel<uint16_t><<<grid_of(B.n), 256, 0, s>>>(P);
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
