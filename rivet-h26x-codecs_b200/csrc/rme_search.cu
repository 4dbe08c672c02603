// The motion search on the device: one persistent launch, one warp per
// (block, reference) task, tasks pulled from a device work queue.
//
// What a task computes is the reference's search, step for step:
//   HEVC   search_full   (encode/h265_me.rs:3749-3858): seeds rounded
//          toward zero (>> 2), clamp_pos to +-(pad - MARGIN), deduplicated
//          through `tried`, scored SAD + (lam * mv_bits) as u32, strict <;
//          then the small diamond (1,0),(-1,0),(0,1),(0,-1) from a fixed
//          `from`, at most 2 * range rounds, inside +-range of the best
//          seed; optional square rings at 4, 8, 16 that restart it.
//          refine_subpel (h265_me.rs:3868-3922): the 3x3 ring at half then
//          at quarter samples (dy outer, dx inner; the cross at quarter
//          samples when asked), SATD + rate, strict <.
//   H.264  Search::int_search (encode/h264_hpel.rs:789-952) and
//          Search::refine (956-1021): predictor plus deduplicated
//          candidates (rounded (m + 2) >> 2, clamped to search_bounds),
//          UMH cross and hexagon rings, small diamond or the hexagon with
//          its three-new-points continuation, the square; half- then
//          quarter-sample rings that skip points within one step of the
//          previous centre; SAD / SATD + MvCostTable rate, strict <.
// The reference scores one candidate at a time; here a warp scores every
// candidate of a step together (they are all known before the step: each
// ring is around a centre fixed for the step) and then accepts them in the
// reference's order with its strict <, so the chosen vector, its cost and
// the candidate counts are the reference's (the sum for a candidate does
// not depend on when it is taken, and a point equal to the current best
// has the best cost, so a strict < never takes it).
//
// Distortion: 8-bit SAD is __vsadu4 over four packed samples, 10/12-bit
// __vsadu2 over two (packed 16-bit lanes); SATD is the 4x4 Hadamard of
// dsp/distortion.rs:326-381 with (sum + 1) >> 1 per tile. H.264 quarter
// samples are __vavgu4 / __vavgu2 of two half-sample plane reads (the
// rounded average of the QPEL table, h264_hpel.rs:205-222); HEVC
// fractional samples are reads of the precomputed phase planes.
//
// Scheduling: in STANDALONE mode a task's seeds come from other tasks'
// results (its left and upper neighbours at the same size, the enclosing
// block one size up; H.264: the A, B, C / D macroblocks). The queue lists
// every frame's tasks in an order where each task comes after everything
// it reads, so a warp that claims a task only ever waits on tasks claimed
// earlier by warps that are running; each wait is bounded (kSpinLimit
// polls with backoff) and a wait that runs out sets a status bit the host
// turns into RME_EDEVICE instead of hanging.
#include <cuda_runtime.h>

#include "rme_internal.h"

namespace rme {
namespace {

constexpr int kMaxBlk = 64;

struct alignas(16) WarpSmem {
  uint32_t src[kMaxBlk * kMaxBlk / 2];  // source block as 32-bit words (row stride w*bytes/4)
  int cx[32], cy[32];                   // candidates of the step
  uint32_t cost[32];                    // their SAD or SATD
  const void* p1[32];                   // SATD: first plane view of each candidate
  const void* p2[32];                   //       second view to average with (H.264), or null
  int tx[16], ty[16];                   // seed staging / tried
  int n;
};

// ---- memory helpers --------------------------------------------------------
__device__ __forceinline__ int ld_acquire(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int32_t* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Four 8-bit or two 16-bit samples starting at any sample address.
__device__ __forceinline__ uint32_t ldw(const uint8_t* p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  uint32_t lo = __ldg(q), hi = __ldg(q + 1);
  return __funnelshift_r(lo, hi, (uint32_t)(a & 3) * 8u);
}
__device__ __forceinline__ uint32_t ldw(const uint16_t* p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  uint32_t lo = __ldg(q), hi = __ldg(q + 1);
  return __funnelshift_r(lo, hi, (uint32_t)(a & 2) * 8u);
}
__device__ __forceinline__ uint32_t vsad(uint32_t a, uint32_t b, uint8_t) { return __vsadu4(a, b); }
__device__ __forceinline__ uint32_t vsad(uint32_t a, uint32_t b, uint16_t) { return __vsadu2(a, b); }
__device__ __forceinline__ uint32_t vavg(uint32_t a, uint32_t b, uint8_t) { return __vavgu4(a, b); }
__device__ __forceinline__ uint32_t vavg(uint32_t a, uint32_t b, uint16_t) { return __vavgu2(a, b); }

// 4x4 Hadamard SATD of one tile (dsp/distortion.rs:326-381).
__device__ __forceinline__ uint32_t satd4x4(int d[16]) {
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

// Lanes per candidate: the largest of 8/4/2/1 (SAD) or 4/2/1 (SATD) that
// divides the candidate's work items, so each lane of a candidate's group
// has the same number of items and a butterfly reduces the group.
__device__ __forceinline__ int lanes_for(int items, int maxl) {
  return (maxl >= 8 && (items & 7) == 0) ? 8 : ((items & 3) == 0 ? 4 : ((items & 1) == 0 ? 2 : 1));
}

// SAD of sm.cx/cy[0..n) (whole-sample offsets from the block at `org`).
template <class S>
__device__ __noinline__ void sad_batch(WarpSmem& sm, const S* org, int stride, int w, int h, int n, int lane) {
  constexpr int SPW = 4 / sizeof(S);
  const int WR = w / SPW, IPC = WR * h;
  const int LPC = lanes_for(IPC, 8), CPP = 32 / LPC, IPL = IPC / LPC;
  const int sub = lane & (LPC - 1), grp = lane / LPC;
  for (int c0 = 0; c0 < n; c0 += CPP) {
    int c = c0 + grp;
    uint32_t acc = 0;
    if (c < n) {
      const S* rp = org + (ptrdiff_t)sm.cy[c] * stride + sm.cx[c];
      int row = sub / WR, wd = sub % WR;
      for (int u = 0; u < IPL; ++u) {
        acc += vsad(sm.src[row * WR + wd], ldw(rp + (ptrdiff_t)row * stride + wd * SPW), S());
        wd += LPC;
        while (wd >= WR) {
          wd -= WR;
          ++row;
        }
      }
    }
    for (int o = LPC >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (sub == 0 && c < n) sm.cost[c] = acc;
  }
  __syncwarp();
}

// SATD of the predictions sm.p1[k] (averaged with sm.p2[k] where set),
// k < n, against the source block.
template <class S>
__device__ __noinline__ void satd_batch(WarpSmem& sm, int stride, int w, int h, int n, int lane) {
  constexpr int SPW = 4 / sizeof(S);
  const int WR = w / SPW, TW = w >> 2, TPC = TW * (h >> 2);
  const int LPC = lanes_for(TPC, 4), CPP = 32 / LPC, IPL = TPC / LPC;
  const int sub = lane & (LPC - 1), grp = lane / LPC;
  for (int c0 = 0; c0 < n; c0 += CPP) {
    int c = c0 + grp;
    uint32_t acc = 0;
    if (c < n) {
      const S* a = (const S*)sm.p1[c];
      const S* b = (const S*)sm.p2[c];
      int ty = sub / TW, tx = sub % TW;
      for (int u = 0; u < IPL; ++u) {
        int d[16];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          ptrdiff_t off = (ptrdiff_t)(ty * 4 + r) * stride + tx * 4;
          const uint32_t* srow = &sm.src[(ty * 4 + r) * WR + tx * (4 / SPW)];
#pragma unroll
          for (int k = 0; k < 4 / SPW; ++k) {
            uint32_t pw = ldw(a + off + k * SPW);
            if (b) pw = vavg(pw, ldw(b + off + k * SPW), S());
            uint32_t sw = srow[k];
#pragma unroll
            for (int e = 0; e < SPW; ++e) {
              int sh = e * (32 / SPW);
              uint32_t m = SPW == 4 ? 0xffu : 0xffffu;
              d[r * 4 + k * SPW + e] = (int)((sw >> sh) & m) - (int)((pw >> sh) & m);
            }
          }
        }
        acc += satd4x4(d);
        tx += LPC;
        while (tx >= TW) {
          tx -= TW;
          ++ty;
        }
      }
    }
    for (int o = LPC >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (sub == 0 && c < n) sm.cost[c] = acc;
  }
  __syncwarp();
}

// The source block into shared memory as words.
template <class S>
__device__ __forceinline__ void stage_src(WarpSmem& sm, const S* org, int stride, int w, int h, int lane) {
  constexpr int SPW = 4 / sizeof(S);
  const int WR = w / SPW;
  __syncwarp();
  for (int i = lane; i < WR * h; i += 32) {
    int row = i / WR, wd = i - row * WR;
    sm.src[i] = ldw(org + (ptrdiff_t)row * stride + wd * SPW);
  }
  __syncwarp();
}

template <class S>
__device__ __forceinline__ const S* plane_at(const DevPlanes& p, int plane, int x, int y) {
  return (const S*)p.base + (int64_t)plane * p.plane_elems + p.origin + (int64_t)y * p.stride + x;
}

// Bounded wait for a dependency's flag (lane 0), then a warp barrier.
__device__ __forceinline__ void wait_flag(const int32_t* f, int epoch, uint32_t* status, int lane) {
  if (lane == 0) {
    uint32_t ns = 32;
    uint32_t it = 0;
    while (ld_acquire(f) != epoch) {
      if (++it >= kSpinLimit) {
        atomicOr(status, kStatusWaitTimeout);
        break;
      }
      __nanosleep(ns);
      if (ns < 1024) ns <<= 1;
    }
  }
  __syncwarp();
}

__device__ __forceinline__ uint32_t ldcg_u32(const void* p) { return __ldcg((const unsigned int*)p); }
__device__ __forceinline__ int mvx_of(uint32_t v) { return (int)(int16_t)(v & 0xffffu); }
__device__ __forceinline__ int mvy_of(uint32_t v) { return (int)(int16_t)(v >> 16); }

struct Counters {
  unsigned long long tasks = 0, sad = 0, satd = 0, sad_samples = 0, satd_samples = 0;
};

__device__ __forceinline__ void write_result(rme_result* o, int mvx, int mvy, int ref, uint32_t cost, uint32_t satd,
                                             int imx, int imy, uint32_t icost, uint32_t nsad, uint32_t nsatd,
                                             int lane) {
  if (lane == 0) {
    rme_result r;
    r.mv.x = (int16_t)mvx;
    r.mv.y = (int16_t)mvy;
    r.ref = ref;
    r.cost = cost;
    r.satd = satd;
    r.int_mv.x = (int16_t)imx;
    r.int_mv.y = (int16_t)imy;
    r.int_cost = icost;
    r.n_sad = nsad;
    r.n_satd = nsatd;
    *o = r;
  }
}

// ---- HEVC -------------------------------------------------------------------

// mvd_component_bits (h265_search.rs:212-247) in closed form: 1 at zero,
// else 3 + 2 * floor(log2 |d|) (the loop of mvd_bits_of counts
// floor(log2 |d|) - 1 Exp-Golomb prefix steps past the first).
__device__ __forceinline__ uint32_t hevc_cbits(int d) {
  uint32_t a = (uint32_t)abs(d);
  return a == 0 ? 1u : 3u + 2u * (31u - __clz(a));
}
__device__ __forceinline__ uint32_t hevc_rate(const FrameDesc& F, int mx, int my, const int pq[4]) {
  uint32_t b0 = hevc_cbits(mx - pq[0]) + hevc_cbits(my - pq[1]);
  uint32_t b1 = hevc_cbits(mx - pq[2]) + hevc_cbits(my - pq[3]);
  uint32_t bits = min(b0, b1) + 1u;
  return __ldg(&F.lam_bits[min(bits, (uint32_t)(kLamBits - 1))]);
}

template <class S>
__device__ void hevc_task(const FrameDesc& F, int t, WarpSmem& sm, int lane, uint32_t* status, Counters& cnt) {
  int r, x, y, w, h, ns;
  int pq[4];
  int32_t* flag = nullptr;
  rme_result* out;
  if (F.mode == RME_PRED_GIVEN) {
    const rme_job* j = &F.jobs[t];
    r = j->ref;
    x = j->x;
    y = j->y;
    w = j->w;
    h = j->h;
    ns = j->nseeds;
    pq[0] = j->mvp[0].x;
    pq[1] = j->mvp[0].y;
    pq[2] = j->mvp[1].x;
    pq[3] = j->mvp[1].y;
    if (lane < ns) {
      sm.tx[lane] = j->seeds[lane].x;
      sm.ty[lane] = j->seeds[lane].y;
    }
    out = &F.out[t];
  } else {
    r = t % F.nref;
    int blk = t / F.nref, l = 0;
    while (l + 1 < F.nlevels && blk >= F.base[l + 1]) ++l;
    int local = blk - F.base[l], nbx = F.nbx[l];
    int by = local / nbx, bx = local - by * nbx, N = F.size[l];
    x = bx * N;
    y = by * N;
    w = h = N;
    // AMVP pair from the left and upper results of this level, the parent
    // seed from the enclosing block one evaluated size up.
    int na = 0, ax = 0, ay = 0, bxv = 0, byv = 0;
    if (bx > 0) {
      int idx = (F.base[l] + local - 1) * F.nref + r;
      wait_flag(&F.flags[idx], F.epoch, status, lane);
      uint32_t v = ldcg_u32(&F.out[idx].mv);
      ax = mvx_of(v);
      ay = mvy_of(v);
      na = 1;
    }
    if (by > 0) {
      int idx = (F.base[l] + local - nbx) * F.nref + r;
      wait_flag(&F.flags[idx], F.epoch, status, lane);
      uint32_t v = ldcg_u32(&F.out[idx].mv);
      int qx = mvx_of(v), qy = mvy_of(v);
      if (na == 0) {
        ax = qx;
        ay = qy;
        na = 1;
      } else if (qx != ax || qy != ay) {
        bxv = qx;
        byv = qy;
        na = 2;
      }
    }
    pq[0] = na > 0 ? ax : 0;
    pq[1] = na > 0 ? ay : 0;
    pq[2] = na > 1 ? bxv : 0;
    pq[3] = na > 1 ? byv : 0;
    ns = 3;
    int psx = 0, psy = 0;
    bool parent = false;
    if (l > 0) {
      int Np = F.size[l - 1], px = x / Np, py = y / Np;
      if (px < F.nbx[l - 1] && py < F.nby[l - 1]) {
        int idx = (F.base[l - 1] + py * F.nbx[l - 1] + px) * F.nref + r;
        wait_flag(&F.flags[idx], F.epoch, status, lane);
        uint32_t v = ldcg_u32(&F.out[idx].mv);
        psx = mvx_of(v);
        psy = mvy_of(v);
        parent = true;
      }
    }
    if (lane == 0) {
      sm.tx[0] = 0;
      sm.ty[0] = 0;
      sm.tx[1] = pq[0];
      sm.ty[1] = pq[1];
      sm.tx[2] = pq[2];
      sm.ty[2] = pq[3];
      sm.tx[3] = psx;
      sm.ty[3] = psy;
    }
    if (parent) ns = 4;
    flag = &F.flags[t];
    out = &F.out[t];
  }
  const DevPlanes& R = F.ref[r];
  const S* src = plane_at<S>(F.src, 0, x, y);
  stage_src(sm, src, F.src.stride, w, h, lane);
  const S* org = plane_at<S>(R, 0, x, y);
  const int stride = R.stride;
  const int padm = F.pad - 4;  // h265_search.rs MARGIN
  const int lox = -padm - x, hix = F.width + padm - w - x, loy = -padm - y, hiy = F.height + padm - h - y;
  uint32_t nsad = 0, nsatd = 0;

  // Seeds: >> 2, clamp_pos, dedupe through tried[16] (h265_me.rs:3785-3800).
  if (lane == 0) {
    int tx[16], ty[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      tx[i] = INT32_MIN;
      ty[i] = 0;
    }
    int n = 0;
    for (int i = 0; i < ns; ++i) {
      int cx = min(max(sm.tx[i] >> 2, lox), hix), cy = min(max(sm.ty[i] >> 2, loy), hiy);
      bool seen = false;
#pragma unroll
      for (int k = 0; k < 16; ++k) seen |= (tx[k] == cx && ty[k] == cy);
      if (seen) continue;
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (k == i) {
          tx[k] = cx;
          ty[k] = cy;
        }
      sm.cx[n] = cx;
      sm.cy[n] = cy;
      ++n;
    }
    sm.n = n;
  }
  __syncwarp();
  int n = sm.n;
  sad_batch<S>(sm, org, stride, w, h, n, lane);
  int bx = 0, by = 0;
  uint32_t bcost = 0xffffffffu;
  for (int k = 0; k < n; ++k) {
    uint32_t c = sm.cost[k] + hevc_rate(F, sm.cx[k] * 4, sm.cy[k] * 4, pq);
    if (c < bcost) {
      bcost = c;
      bx = sm.cx[k];
      by = sm.cy[k];
    }
  }
  nsad += n;
  const int ox = bx, oy = by, range = F.search_range;
  auto inside = [&](int cx, int cy) {
    return abs(cx - ox) <= range && abs(cy - oy) <= range && cx >= lox && cx <= hix && cy >= loy && cy <= hiy;
  };
  int rings = 0;
  for (;;) {
    for (int it = 0; it < 2 * range; ++it) {
      int fx = bx, fy = by;
      __syncwarp();
      // Lanes 0..3 each own one diamond point; the valid ones are packed
      // in order.
      int dxs = lane == 0 ? 1 : lane == 1 ? -1 : 0, dys = lane == 2 ? 1 : lane == 3 ? -1 : 0;
      bool ok = lane < 4 && inside(fx + dxs, fy + dys);
      uint32_t m = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        int pos = __popc(m & ((1u << lane) - 1));
        sm.cx[pos] = fx + dxs;
        sm.cy[pos] = fy + dys;
      }
      __syncwarp();
      int nd = __popc(m);
      sad_batch<S>(sm, org, stride, w, h, nd, lane);
      bool improved = false;
      for (int k = 0; k < nd; ++k) {
        uint32_t c = sm.cost[k] + hevc_rate(F, sm.cx[k] * 4, sm.cy[k] * 4, pq);
        if (c < bcost) {
          bcost = c;
          bx = sm.cx[k];
          by = sm.cy[k];
          improved = true;
        }
      }
      nsad += nd;
      if (!improved) break;
    }
    if (rings >= F.search_rings) break;
    ++rings;
    int fx = bx, fy = by;
    __syncwarp();
    // Square rings at 4, 8, 16: 24 points, in the reference's order.
    int rr = lane < 8 ? 4 : lane < 16 ? 8 : 16, k8 = lane & 7;
    int dxs = (k8 == 0 || k8 == 4 || k8 == 6) ? rr : (k8 == 1 || k8 == 5 || k8 == 7) ? -rr : 0;
    int dys = (k8 == 2 || k8 == 4 || k8 == 5) ? rr : (k8 == 3 || k8 == 6 || k8 == 7) ? -rr : 0;
    bool ok = lane < 24 && inside(fx + dxs, fy + dys);
    uint32_t m = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      int pos = __popc(m & ((1u << lane) - 1));
      sm.cx[pos] = fx + dxs;
      sm.cy[pos] = fy + dys;
    }
    __syncwarp();
    int nr = __popc(m);
    sad_batch<S>(sm, org, stride, w, h, nr, lane);
    bool moved = false;
    for (int k = 0; k < nr; ++k) {
      uint32_t c = sm.cost[k] + hevc_rate(F, sm.cx[k] * 4, sm.cy[k] * 4, pq);
      if (c < bcost) {
        bcost = c;
        bx = sm.cx[k];
        by = sm.cy[k];
        moved = true;
      }
    }
    nsad += nr;
    if (!moved) break;
  }
  const uint32_t int_cost = bcost;
  const int imx = bx * 4, imy = by * 4;

  // refine_subpel: the start and the half-sample ring in one batch, then
  // the quarter-sample ring around the winner.
  auto set_cand = [&](int k, int mx, int my) {
    sm.cx[k] = mx;
    sm.cy[k] = my;
    sm.p1[k] = plane_at<S>(R, (my & 3) * 4 + (mx & 3), x + (mx >> 2), y + (my >> 2));
    sm.p2[k] = nullptr;
  };
  __syncwarp();
  if (lane < 9) {
    // k = 0: the start; k = 1..8: dy in {-2,0,2} outer, dx inner, centre skipped.
    int q = lane == 0 ? 4 : (lane <= 4 ? lane - 1 : lane);
    set_cand(lane, imx + (q % 3 - 1) * 2, imy + (q / 3 - 1) * 2);
  }
  __syncwarp();
  satd_batch<S>(sm, stride, w, h, 9, lane);
  int bmx = imx, bmy = imy;
  uint32_t bsatd = sm.cost[0];
  uint32_t bc = bsatd + hevc_rate(F, imx, imy, pq);
  for (int k = 1; k < 9; ++k) {
    uint32_t c = sm.cost[k] + hevc_rate(F, sm.cx[k], sm.cy[k], pq);
    if (c < bc) {
      bc = c;
      bsatd = sm.cost[k];
      bmx = sm.cx[k];
      bmy = sm.cy[k];
    }
  }
  nsatd += 9;
  {
    int cmx = bmx, cmy = bmy;
    __syncwarp();
    bool cross = F.quarter_cross != 0;
    int q = lane < 4 ? lane : lane + 1;  // ring positions 0..8 minus the centre
    int dx = q % 3 - 1, dy = q / 3 - 1;
    bool ok = lane < 8 && !(cross && dx != 0 && dy != 0);
    uint32_t m = __ballot_sync(0xffffffffu, ok);
    if (ok) set_cand(__popc(m & ((1u << lane) - 1)), (int)(int16_t)(cmx + dx), (int)(int16_t)(cmy + dy));
    __syncwarp();
    int nq = __popc(m);
    satd_batch<S>(sm, stride, w, h, nq, lane);
    for (int k = 0; k < nq; ++k) {
      uint32_t c = sm.cost[k] + hevc_rate(F, sm.cx[k], sm.cy[k], pq);
      if (c < bc) {
        bc = c;
        bsatd = sm.cost[k];
        bmx = sm.cx[k];
        bmy = sm.cy[k];
      }
    }
    nsatd += nq;
  }
  write_result(out, bmx, bmy, r, bc, bsatd, imx, imy, int_cost, nsad, nsatd, lane);
  if (flag) {
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release(flag, F.epoch);
    }
  }
  cnt.tasks += 1;
  cnt.sad += nsad;
  cnt.satd += nsatd;
  cnt.sad_samples += (unsigned long long)nsad * w * h;
  cnt.satd_samples += (unsigned long long)nsatd * w * h;
}

// ---- H.264 ------------------------------------------------------------------

__constant__ int8_t c_h264_qpel[16][6] = {
    {0, 0, 0, -1, 0, 0}, {0, 0, 0, 1, 0, 0}, {1, 0, 0, -1, 0, 0}, {1, 0, 0, 0, 1, 0},
    {0, 0, 0, 2, 0, 0},  {1, 0, 0, 2, 0, 0}, {1, 0, 0, 3, 0, 0},  {1, 0, 0, 2, 1, 0},
    {2, 0, 0, -1, 0, 0}, {2, 0, 0, 3, 0, 0}, {3, 0, 0, -1, 0, 0}, {3, 0, 0, 2, 1, 0},
    {2, 0, 0, 0, 0, 1},  {2, 0, 0, 1, 0, 1}, {3, 0, 0, 1, 0, 1},  {2, 1, 0, 1, 0, 1},
};
__constant__ int8_t c_hex[6][2] = {{-2, 0}, {-1, -2}, {1, -2}, {2, 0}, {1, 2}, {-1, 2}};
__constant__ int8_t c_sq[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
__constant__ int8_t c_ring[8][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
__constant__ int8_t c_hex12[12][2] = {{-2, 1}, {-2, -1}, {2, 1},  {2, -1}, {-1, 2},  {1, 2},
                                      {-1, -2}, {1, -2}, {-2, 2}, {2, 2},  {-2, -2}, {2, -2}};

struct H264Blk {
  int x, y, w, h;
  int px, py;       // predictor (quarter samples)
  int lx, hx, ly, hy;  // search_bounds
};

__device__ __forceinline__ uint32_t h264_rate(const FrameDesc& F, const H264Blk& B, int qx, int qy) {
  int dx = min(max(qx - B.px, -kMvSpan), kMvSpan), dy = min(max(qy - B.py, -kMvSpan), kMvSpan);
  return (uint32_t)__ldg(&F.tab[dx + kMvSpan]) + (uint32_t)__ldg(&F.tab[dy + kMvSpan]);
}

// ring(): points around a fixed centre c (offsets from `offs` of length
// nof, lane k owns offset k), inside the box and not the centre, scored
// together, accepted in order; returns the offset index of the last
// point taken or -1.
template <class S>
__device__ int h264_ring(const FrameDesc& F, const H264Blk& B, WarpSmem& sm, const S* org, int stride, int lane,
                         int cx, int cy, int ox, int oy, bool valid_lane, int box[4], int& bx, int& by,
                         uint32_t& bcost, uint32_t& nsad) {
  __syncwarp();
  int fx = cx + ox, fy = cy + oy;
  bool ok = valid_lane && fx >= box[0] && fx <= box[1] && fy >= box[2] && fy <= box[3] && !(fx == cx && fy == cy);
  uint32_t m = __ballot_sync(0xffffffffu, ok);
  if (ok) {
    int pos = __popc(m & ((1u << lane) - 1));
    sm.cx[pos] = fx;
    sm.cy[pos] = fy;
    sm.tx[pos] = lane;
  }
  __syncwarp();
  int n = __popc(m);
  sad_batch<S>(sm, org, stride, B.w, B.h, n, lane);
  int moved = -1;
  for (int k = 0; k < n; ++k) {
    uint32_t c = sm.cost[k] + h264_rate(F, B, sm.cx[k] * 4, sm.cy[k] * 4);
    if (c < bcost) {
      bcost = c;
      bx = sm.cx[k];
      by = sm.cy[k];
      moved = sm.tx[k];
    }
  }
  nsad += n;
  return moved;
}

// Search::int_search (h264_hpel.rs:789-952) for one reference: lane k
// holds candidate k of `ncand` (quarter samples).
template <class S>
__device__ void h264_int_search(const FrameDesc& F, const H264Blk& B, WarpSmem& sm, int lane, const DevPlanes& R,
                                int ncand, int cand_x, int cand_y, int& imx, int& imy, uint32_t& icost,
                                uint32_t& nsad) {
  const S* org = plane_at<S>(R, 0, B.x, B.y);
  const int stride = R.stride;
  auto clampf = [&](int m, int lo, int hi) { return min(max((m + 2) >> 2, lo), hi); };
  int bx = clampf(B.px, B.lx, B.hx), by = clampf(B.py, B.ly, B.hy);
  // The predictor and the distinct candidates (tried[12]), in order.
  __syncwarp();
  int fx = clampf(cand_x, B.lx, B.hx), fy = clampf(cand_y, B.ly, B.hy);
  if (lane < ncand) {
    sm.tx[lane] = fx;
    sm.ty[lane] = fy;
  }
  __syncwarp();
  if (lane == 0) {
    int tx[12], ty[12], nt = 0, n = 1;
    sm.cx[0] = bx;
    sm.cy[0] = by;
    for (int i = 0; i < ncand; ++i) {
      int qx = sm.tx[i], qy = sm.ty[i];
      bool seen = qx == bx && qy == by;
      for (int k = 0; k < nt; ++k) seen |= (tx[k] == qx && ty[k] == qy);
      if (seen) continue;
      if (nt < 12) {
        tx[nt] = qx;
        ty[nt] = qy;
        ++nt;
      }
      sm.cx[n] = qx;
      sm.cy[n] = qy;
      ++n;
    }
    sm.n = n;
  }
  __syncwarp();
  int n = sm.n;
  sad_batch<S>(sm, org, stride, B.w, B.h, n, lane);
  uint32_t bcost = sm.cost[0] + h264_rate(F, B, bx * 4, by * 4);
  for (int k = 1; k < n; ++k) {
    uint32_t c = sm.cost[k] + h264_rate(F, B, sm.cx[k] * 4, sm.cy[k] * 4);
    if (c < bcost) {
      bcost = c;
      bx = sm.cx[k];
      by = sm.cy[k];
    }
  }
  nsad += n;
  const int range = F.range;
  int box[4] = {max(bx - range, B.lx), min(bx + range, B.hx), max(by - range, B.ly), min(by + range, B.hy)};
  if (F.umh) {
    // The cross r = 2, 4, .. range then 12-point hexagon rings r = 4, 8, ..
    // range around the fixed start, each point taken by try_at: skipped
    // when outside the box or equal to the best so far, else scored.
    const int cx = bx, cy = by;
    const int ncross = 4 * (range / 2), nhex = 12 * (range / 4), total = ncross + nhex;
    for (int c0 = 0; c0 < total; c0 += 32) {
      __syncwarp();
      int i = c0 + lane, qx = 0, qy = 0;
      bool ok = i < total;
      if (ok) {
        if (i < ncross) {
          int rr = 2 * (i / 4 + 1), k = i & 3;
          qx = cx + (k == 0 ? -rr : k == 1 ? rr : 0);
          qy = cy + (k == 2 ? -rr : k == 3 ? rr : 0);
        } else {
          int j = i - ncross, rr = 4 * (j / 12 + 1), k = j % 12;
          qx = cx + c_hex12[k][0] * rr / 2;
          qy = cy + c_hex12[k][1] * rr / 2;
        }
        ok = qx >= box[0] && qx <= box[1] && qy >= box[2] && qy <= box[3];
      }
      uint32_t m = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        int pos = __popc(m & ((1u << lane) - 1));
        sm.cx[pos] = qx;
        sm.cy[pos] = qy;
      }
      __syncwarp();
      int nb = __popc(m);
      sad_batch<S>(sm, org, stride, B.w, B.h, nb, lane);
      for (int k = 0; k < nb; ++k) {
        if (sm.cx[k] == bx && sm.cy[k] == by) continue;
        ++nsad;
        uint32_t c = sm.cost[k] + h264_rate(F, B, sm.cx[k] * 4, sm.cy[k] * 4);
        if (c < bcost) {
          bcost = c;
          bx = sm.cx[k];
          by = sm.cy[k];
        }
      }
    }
  }
  if (F.dia) {
    for (int it = 0; it < range; ++it) {
      int cx = bx, cy = by;
      int ox = lane == 0 ? -1 : lane == 1 ? 1 : 0, oy = lane == 2 ? -1 : lane == 3 ? 1 : 0;
      h264_ring<S>(F, B, sm, org, stride, lane, cx, cy, ox, oy, lane < 4, box, bx, by, bcost, nsad);
      if (bx == cx && by == cy) break;
    }
  } else {
    int cx = bx, cy = by;
    int k6 = lane < 6 ? lane : 0;
    int dir = h264_ring<S>(F, B, sm, org, stride, lane, cx, cy, c_hex[k6][0], c_hex[k6][1], lane < 6, box, bx, by,
                           bcost, nsad);
    int it = 1;
    while (dir != -1 && it < range) {
      cx = bx;
      cy = by;
      int ks = lane == 0 ? (dir + 5) % 6 : lane == 1 ? dir : (dir + 1) % 6;
      int moved = h264_ring<S>(F, B, sm, org, stride, lane, cx, cy, c_hex[ks][0], c_hex[ks][1], lane < 3, box, bx,
                               by, bcost, nsad);
      if (moved == -1) {
        dir = -1;
      } else {
        dir = moved == 0 ? (dir + 5) % 6 : moved == 1 ? dir : (dir + 1) % 6;
      }
      ++it;
    }
    cx = bx;
    cy = by;
    int k8 = lane & 7;
    h264_ring<S>(F, B, sm, org, stride, lane, cx, cy, c_sq[k8][0], c_sq[k8][1], lane < 8, box, bx, by, bcost, nsad);
  }
  imx = bx * 4;
  imy = by * 4;
  icost = bcost;
}

// Search::refine (h264_hpel.rs:956-1021) from (smx, smy): the start, then
// `hpel` rings of half-sample points and `qpel` of quarter-sample points
// (the start scored in the same batch as the first ring).
template <class S>
__device__ void h264_refine(const FrameDesc& F, const H264Blk& B, WarpSmem& sm, int lane, const DevPlanes& R, int smx,
                            int smy, int hpel, int qpel, int& omx, int& omy, uint32_t& osatd, uint32_t& ocost,
                            uint32_t& nsatd) {
  const int qlx = B.lx * 4, qhx = B.hx * 4, qly = B.ly * 4, qhy = B.hy * 4;
  auto set_cand = [&](int k, int mx, int my) {
    int xi = B.x + (mx >> 2), yi = B.y + (my >> 2);
    const int8_t* q = c_h264_qpel[(my & 3) * 4 + (mx & 3)];
    sm.cx[k] = mx;
    sm.cy[k] = my;
    sm.p1[k] = plane_at<S>(R, q[0], xi + q[1], yi + q[2]);
    sm.p2[k] = q[3] < 0 ? nullptr : plane_at<S>(R, q[3], xi + q[4], yi + q[5]);
  };
  int bmx = smx, bmy = smy;
  uint32_t bsatd = 0, bc = 0;
  bool first = true;
  for (int s = 0; s < 2; ++s) {
    const int step = s == 0 ? 2 : 1, iters = s == 0 ? hpel : qpel;
    const int pts = (step == 1 && F.qpel_diamond) ? 4 : 8;
    bool has_prev = false;
    int prevx = 0, prevy = 0;
    for (int it = 0; it < iters || first; ++it) {
      const int cmx = bmx, cmy = bmy;
      const bool ring = it < iters;
      __syncwarp();
      // slot 0: the start (first batch only); then the ring's points.
      const int base = first ? 1 : 0;
      const int kk = lane & 7;
      const int mx = (int)(int16_t)(cmx + c_ring[kk][0] * step), my = (int)(int16_t)(cmy + c_ring[kk][1] * step);
      const bool ok = ring && lane < pts && mx >= qlx && mx <= qhx && my >= qly && my <= qhy &&
                      !(has_prev && abs(mx - prevx) <= step && abs(my - prevy) <= step);
      const uint32_t m = __ballot_sync(0xffffffffu, ok);
      if (ok) set_cand(base + __popc(m & ((1u << lane) - 1)), mx, my);
      if (first && lane == 31) set_cand(0, cmx, cmy);
      __syncwarp();
      const int nr = __popc(m), ntot = base + nr;
      satd_batch<S>(sm, R.stride, B.w, B.h, ntot, lane);
      if (first) {
        bsatd = sm.cost[0];
        bc = bsatd + h264_rate(F, B, cmx, cmy);
      }
      for (int k = base; k < ntot; ++k) {
        uint32_t c = sm.cost[k] + h264_rate(F, B, sm.cx[k], sm.cy[k]);
        if (c < bc) {
          bc = c;
          bsatd = sm.cost[k];
          bmx = sm.cx[k];
          bmy = sm.cy[k];
        }
      }
      nsatd += ntot;
      first = false;
      if (!ring) break;
      if (bmx == cmx && bmy == cmy) break;
      prevx = cmx;
      prevy = cmy;
      has_prev = true;
    }
  }
  omx = bmx;
  omy = bmy;
  osatd = bsatd;
  ocost = bc;
}

// median_mvp (h264/mb.rs:1170-1189) over (avail, ref, mv) neighbours.
struct Nb {
  bool avail;
  int ref, x, y;
};
__device__ __forceinline__ int med3(int a, int b, int c) { return min(max(a, b), max(min(a, b), c)); }
__device__ __forceinline__ void median_mvp(Nb a, Nb b, Nb c, int ref, int& ox, int& oy) {
  if (!b.avail && !c.avail && a.avail) {
    b = a;
    c = a;
  }
  bool ma = a.ref == ref, mb = b.ref == ref, mc = c.ref == ref;
  if (ma && !mb && !mc) {
    ox = a.x;
    oy = a.y;
  } else if (!ma && mb && !mc) {
    ox = b.x;
    oy = b.y;
  } else if (!ma && !mb && mc) {
    ox = c.x;
    oy = c.y;
  } else {
    ox = med3(a.x, b.x, c.x);
    oy = med3(a.y, b.y, c.y);
  }
}

template <class S>
__device__ void h264_task(const FrameDesc& F, int t, WarpSmem& sm, int lane, uint32_t* status, Counters& cnt) {
  H264Blk B;
  uint32_t nsad = 0, nsatd = 0;
  auto bounds = [&](int x, int y, int w, int h) {  // search_bounds (h264_hpel.rs:476-488)
    B.lx = 4 - F.pad - x;
    B.hx = F.width + F.pad - (w + 4) - x;
    B.ly = max(4 - F.pad - y, -F.vr);
    B.hy = min(F.height + F.pad - (h + 4) - y, F.vr);
  };
  if (F.mode == RME_PRED_GIVEN) {
    const rme_job* j = &F.jobs[t];
    B.x = j->x;
    B.y = j->y;
    B.w = j->w;
    B.h = j->h;
    B.px = j->mvp[0].x;
    B.py = j->mvp[0].y;
    bounds(B.x, B.y, B.w, B.h);
    int nc = j->nseeds;
    int cx = lane < nc ? j->seeds[lane].x : 0, cy = lane < nc ? j->seeds[lane].y : 0;
    stage_src(sm, plane_at<S>(F.src, 0, B.x, B.y), F.src.stride, B.w, B.h, lane);
    int mx, my, imx, imy;
    uint32_t sat, c, ic;
    const bool score = (j->flags & RME_JOB_SCORE_ONLY) != 0;
    h264_int_search<S>(F, B, sm, lane, F.ref[j->ref], nc, cx, cy, imx, imy, ic, nsad);
    h264_refine<S>(F, B, sm, lane, F.ref[j->ref], imx, imy, score ? 0 : F.hpel_iters, score ? 0 : F.qpel_iters, mx, my,
                   sat, c, nsatd);
    write_result(&F.out[t], mx, my, j->ref, c, sat, imx, imy, ic, nsad, nsatd, lane);
  } else {
    // p_mb's search section (h264_analyse.rs:1884-1975) with the
    // neighbours' final 16x16 results as the motion context.
    const int mbw = F.width / 16, mx = t % mbw, my = t / mbw;
    B.x = mx * 16;
    B.y = my * 16;
    B.w = B.h = 16;
    bounds(B.x, B.y, 16, 16);
    auto nb = [&](int qx, int qy) {
      Nb m{false, -1, 0, 0};
      if (qx < 0 || qy < 0 || qx >= mbw) return m;
      int idx = qy * mbw + qx;
      wait_flag(&F.flags[idx], F.epoch, status, lane);
      uint32_t v = ldcg_u32(&F.out[idx].mv);
      m.avail = true;
      m.ref = (int)ldcg_u32(&F.out[idx].ref);
      m.x = mvx_of(v);
      m.y = mvy_of(v);
      return m;
    };
    Nb A = nb(mx - 1, my), Bn = nb(mx, my - 1), C = nb(mx + 1, my - 1), D = nb(mx - 1, my - 1);
    Nb Cc = C.avail ? C : D;
    // p_skip_mv (h264/mb.rs:1235-1246)
    int skx = 0, sky = 0;
    if (A.avail && Bn.avail && !(A.ref == 0 && A.x == 0 && A.y == 0) && !(Bn.ref == 0 && Bn.x == 0 && Bn.y == 0))
      median_mvp(A, Bn, Cc, 0, skx, sky);
    // cands = [skip_mv, 0, distinct A, B, C vectors] (h264_pic.rs:713-751)
    int ncx[8], ncy[8], nc = 0;
    ncx[nc] = skx;
    ncy[nc++] = sky;
    ncx[nc] = 0;
    ncy[nc++] = 0;
    {
      Nb q[3] = {A, Bn, C};
      int vx[4], vy[4], nn = 0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        if (!q[i].avail || q[i].ref < 0 || nn >= 4) continue;
        bool dup = false;
        for (int k = 0; k < nn; ++k) dup |= (vx[k] == q[i].x && vy[k] == q[i].y);
        if (!dup) {
          vx[nn] = q[i].x;
          vy[nn++] = q[i].y;
        }
      }
      for (int k = 0; k < nn; ++k) {
        ncx[nc] = vx[k];
        ncy[nc++] = vy[k];
      }
    }
    stage_src(sm, plane_at<S>(F.src, 0, B.x, B.y), F.src.stride, 16, 16, lane);
    int mv16x = 0, mv16y = 0, r16 = 0, mi16x = 0, mi16y = 0;
    uint32_t c16 = 0xffffffffu, s16 = 0, ci16 = 0, int16 = 0xffffffffu;
    for (int r = 0; r < F.nref; ++r) {
      int prx, pry;
      median_mvp(A, Bn, Cc, r, prx, pry);
      if (r > 0 && nc < 8) {
        ncx[nc] = prx;
        ncy[nc] = pry;
      }
      int k = r > 0 ? min(nc + 1, 8) : nc;
      B.px = prx;
      B.py = pry;
      int cx = 0, cy = 0;
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (lane == i) {
          cx = ncx[i];
          cy = ncy[i];
        }
      int mx2, my2, imx, imy;
      uint32_t sat, c, ci;
      h264_int_search<S>(F, B, sm, lane, F.ref[r], k, cx, cy, imx, imy, ci, nsad);
      ci += F.ref_cost[r];
      // refine_ratio: a further reference whose whole-sample cost is that
      // factor of the best so far is only scored, not refined (f32 compare,
      // round to nearest, as p_mb's `ci as f32 >= ratio * int16 as f32`).
      const bool gate = r > 0 && F.refine_ratio > 0.0f &&
                        __uint2float_rn(ci) >= __fmul_rn(F.refine_ratio, __uint2float_rn(int16));
      h264_refine<S>(F, B, sm, lane, F.ref[r], imx, imy, gate ? 0 : F.hpel_iters, gate ? 0 : F.qpel_iters, mx2, my2,
                     sat, c, nsatd);
      int16 = min(int16, ci);
      c += F.ref_cost[r];
      if (c < c16) {
        c16 = c;
        mv16x = mx2;
        mv16y = my2;
        s16 = sat;
        r16 = r;
        mi16x = imx;
        mi16y = imy;
        ci16 = ci;
      }
    }
    write_result(&F.out[t], mv16x, mv16y, r16, c16, s16, mi16x, mi16y, ci16, nsad, nsatd, lane);
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release(&F.flags[t], F.epoch);
    }
  }
  cnt.tasks += 1;
  cnt.sad += nsad;
  cnt.satd += nsatd;
  cnt.sad_samples += (unsigned long long)nsad * B.w * B.h;
  cnt.satd_samples += (unsigned long long)nsatd * B.w * B.h;
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32) search_kernel(LaunchDesc L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& sm = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
  Counters cnt;
  for (;;) {
    unsigned long long g = 0;
    if (lane == 0) g = atomicAdd(L.head, 1ull);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= (unsigned long long)L.total) break;
    uint32_t e = __ldg(&L.queue[g]);
    const FrameDesc& F = L.frames[e >> 24];
    int t = (int)(e & 0xffffffu);
    if (t >= F.ntasks) {
      if (lane == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    }
    if (F.codec == RME_CODEC_HEVC) {
      if (F.bd == 8) hevc_task<uint8_t>(F, t, sm, lane, L.status, cnt);
      else hevc_task<uint16_t>(F, t, sm, lane, L.status, cnt);
    } else {
      if (F.bd == 8) h264_task<uint8_t>(F, t, sm, lane, L.status, cnt);
      else h264_task<uint16_t>(F, t, sm, lane, L.status, cnt);
    }
  }
  if (lane == 0) {
    atomicAdd(&L.counters[0], cnt.tasks);
    atomicAdd(&L.counters[1], cnt.sad);
    atomicAdd(&L.counters[2], cnt.satd);
    atomicAdd(&L.counters[3], cnt.sad_samples);
    atomicAdd(&L.counters[4], cnt.satd_samples);
  }
}

}  // namespace

int search_blocks_per_sm(int) {
  int n = 0;
  size_t smem = sizeof(WarpSmem) * kWarpsPerBlock;
  if (cudaFuncSetAttribute(search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, search_kernel, kWarpsPerBlock * 32, smem) != cudaSuccess)
    return 1;
  return n;
}

cudaError_t launch_search(const LaunchDesc& L, int, int grid, cudaStream_t s) {
  size_t smem = sizeof(WarpSmem) * kWarpsPerBlock;
  cudaError_t e = cudaFuncSetAttribute(search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  search_kernel<<<grid, kWarpsPerBlock * 32, smem, s>>>(L);
  return cudaGetLastError();
}

}  // namespace rme
