// The search's device code, shared by the batched kernels (rme_search.cu)
// and the resident engine (rme_engine.cu): the task functions, the
// distortion and interpolation-plane reads, the dataflow queue. Each file
// includes it into its own anonymous namespace. Reads of pictures go
// through RME_LD32: the read-only cache path in the batched kernels (a
// launch's pictures do not change while it runs); in the engine, where
// picture slots are refilled while the kernel runs, ordinary cached loads,
// which the memory model keeps fresh: a frame's pictures are written before
// its entries are released into the ring, the warp or CTA that takes an
// entry acquires it (then synchronises its threads) before any read, and a
// slot is refilled only after every frame reading it has completed.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "rme_internal.h"

#ifdef RME_PICTURES_CHANGE_IN_FLIGHT
#define RME_LD32(p) __ldca(p)
#else
#define RME_LD32(p) __ldg(p)
#endif

namespace rme {
namespace {



constexpr int kMaxBlk = 64;
constexpr uint32_t kInf = 0xffffffffu;
constexpr unsigned kFull = 0xffffffffu;

// A warp's shared memory. The fixed-size fields come first, so the 8-bit
// view of a 16-bit warp's memory (the resident engine runs both) keeps them
// at the same place.
template <class S>
struct alignas(16) WarpSmem {
  unsigned long long cnt[6];                        // tasks, SAD / SATD candidates and samples
  int ux[32], uy[32];                               // UMH candidates of a pass (in-order counting)
  uint32_t uc[32];
  uint32_t src[kMaxBlk * kMaxBlk * sizeof(S) / 4];  // source block as words, row stride w*sizeof(S)/4
};
static_assert(offsetof(WarpSmem<uint8_t>, src) == offsetof(WarpSmem<uint16_t>, src), "shared header layout");
static_assert(offsetof(WarpSmem<uint8_t>, src) % 16 == 0, "source block alignment");

// ---- memory helpers --------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Decrement with acquire-release order: the decrement that reaches zero
// has observed every earlier decrementer's writes (their results), and its
// push publishes them all to the task's popper.
__device__ __forceinline__ int dec_acq_rel(int32_t* p) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], -1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}

// Four 8-bit or two 16-bit samples starting at any sample address.
__device__ __forceinline__ uint32_t ldw(const uint8_t* p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  uint32_t lo = RME_LD32(q), hi = RME_LD32(q + 1);
  return __funnelshift_r(lo, hi, (uint32_t)(a & 3) * 8u);
}
__device__ __forceinline__ uint32_t ldw(const uint16_t* p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  uint32_t lo = RME_LD32(q), hi = RME_LD32(q + 1);
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

// Lanes per candidate for a step of n candidates: as many candidates per
// pass as the step has (one pass when n <= 32), at most 32 lanes each.
__device__ __forceinline__ int lanes_per(int n) { return n >= 32 ? 1 : 32 / max(n, 1); }

// The sum over a group of `lpc` consecutive lanes (any width), in every
// lane of the group.
__device__ __forceinline__ uint32_t group_sum(uint32_t v, int lpc, int sub, int lane) {
  for (int o = 1; o < lpc; o <<= 1) {
    const uint32_t t = __shfl_down_sync(kFull, v, o);
    if (sub + o < lpc) v += t;
  }
  return __shfl_sync(kFull, v, lane - sub);
}

// The warp's least cost and the lowest lane holding it. Lanes of one
// candidate group hold the same cost, so that lane is the first lane of
// the first candidate (in the step's order) reaching the least cost.
struct Pick {
  uint32_t cost;
  int lane;
};
__device__ __forceinline__ Pick warp_min(uint32_t cost) {
  uint32_t m = __reduce_min_sync(kFull, cost);
  int l = __ffs(__ballot_sync(kFull, cost == m)) - 1;
  return {m, l};
}

// N consecutive 32-bit words of samples starting at any sample address
// (N + 1 aligned loads, all issued before any is used).
template <int N>
__device__ __forceinline__ void ldwords(const void* p, uint32_t (&out)[N]) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = (uint32_t)(a & 3) * 8u;
  uint32_t w[N + 1];
#pragma unroll
  for (int i = 0; i <= N; ++i) w[i] = RME_LD32(q + i);
#pragma unroll
  for (int i = 0; i < N; ++i) out[i] = __funnelshift_r(w[i], w[i + 1], sh);
}

// SAD of the candidate at whole-sample offset (fx, fy), split over the
// group's lanes in chunks of CW words of a row, summed over the group.
template <class S, int CW>
__device__ __forceinline__ uint32_t sad_chunks(const uint32_t* src, int wr, int h, const S* rp, int stride, int lpc,
                                               int sub) {
  constexpr int SPW = 4 / sizeof(S);
  const int nch = wr / CW, items = nch * h, rs = lpc / nch, cs = lpc % nch;
  int row = sub / nch, col = sub % nch;
  uint32_t acc = 0;
  for (int i = sub; i < items; i += 2 * lpc) {
    uint32_t a[CW], b[CW];
    const int row2 = row + rs + (col + cs >= nch), col2 = (col + cs >= nch) ? col + cs - nch : col + cs;
    const bool two = i + lpc < items;
    ldwords<CW>(rp + (ptrdiff_t)row * stride + col * CW * SPW, a);
    if (two) ldwords<CW>(rp + (ptrdiff_t)row2 * stride + col2 * CW * SPW, b);
#pragma unroll
    for (int k = 0; k < CW; ++k) acc += vsad(src[row * wr + col * CW + k], a[k], S());
    if (two) {
#pragma unroll
      for (int k = 0; k < CW; ++k) acc += vsad(src[row2 * wr + col2 * CW + k], b[k], S());
    }
    row = row2 + rs;
    col = col2 + cs;
    if (col >= nch) {
      col -= nch;
      ++row;
    }
  }
  return acc;
}

template <class S>
__device__ __forceinline__ uint32_t group_sad(const uint32_t* src, int wr, int h, const S* org, int stride, int lpc,
                                              int sub, int lane, bool ok, int fx, int fy) {
  uint32_t acc = 0;
  if (ok) {
    const S* rp = org + (ptrdiff_t)fy * stride + fx;
    if ((wr & 3) == 0) acc = sad_chunks<S, 4>(src, wr, h, rp, stride, lpc, sub);
    else if ((wr & 1) == 0) acc = sad_chunks<S, 2>(src, wr, h, rp, stride, lpc, sub);
    else acc = sad_chunks<S, 1>(src, wr, h, rp, stride, lpc, sub);
  }
  return group_sum(acc, lpc, sub, lane);
}

// SATD over strips of TS horizontally adjacent 4x4 tiles: the strip's four
// rows of prediction samples are loaded (and averaged, H.264) first, then
// each tile's Hadamard.
template <class S, int TS>
__device__ __forceinline__ uint32_t satd_strips(const uint32_t* src, int wr, int tw, int th, const S* p1,
                                                const S* p2, int stride, int lpc, int sub) {
  constexpr int SPW = 4 / sizeof(S);
  constexpr int WPT = 4 / SPW;       // words per tile row
  constexpr int WPS = TS * WPT;      // words per strip row
  const int nspr = tw / TS, items = nspr * th;
  uint32_t acc = 0;
  for (int i = sub; i < items; i += lpc) {
    const int ty = i / nspr, sx = i - ty * nspr;
    uint32_t pw[4][WPS];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const ptrdiff_t off = (ptrdiff_t)(ty * 4 + r) * stride + sx * TS * 4;
      ldwords<WPS>(p1 + off, pw[r]);
      if (p2) {
        uint32_t q[WPS];
        ldwords<WPS>(p2 + off, q);
#pragma unroll
        for (int k = 0; k < WPS; ++k) pw[r][k] = vavg(pw[r][k], q[k], S());
      }
    }
#pragma unroll
    for (int t = 0; t < TS; ++t) {
      int d[16];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const uint32_t* srow = &src[(ty * 4 + r) * wr + (sx * TS + t) * WPT];
#pragma unroll
        for (int k = 0; k < WPT; ++k) {
          const uint32_t sw = srow[k], qw = pw[r][t * WPT + k];
#pragma unroll
          for (int e = 0; e < SPW; ++e) {
            const int sh = e * (32 / SPW);
            const uint32_t m = SPW == 4 ? 0xffu : 0xffffu;
            d[r * 4 + k * SPW + e] = (int)((sw >> sh) & m) - (int)((qw >> sh) & m);
          }
        }
      }
      acc += satd4x4(d);
    }
  }
  return acc;
}

template <class S>
__device__ __forceinline__ uint32_t group_satd(const uint32_t* src, int wr, int tw, int th, const S* p1, const S* p2,
                                               int stride, int lpc, int sub, int lane, bool ok) {
  // Strips of 16 bytes of prediction per row (four 8-bit tiles, two
  // 16-bit ones) where the block is that wide.
  constexpr int TSW = sizeof(S) == 1 ? 4 : 2;
  uint32_t acc = 0;
  if (ok) {
    if (tw % TSW == 0) acc = satd_strips<S, TSW>(src, wr, tw, th, p1, p2, stride, lpc, sub);
    else if ((tw & 1) == 0) acc = satd_strips<S, 2>(src, wr, tw, th, p1, p2, stride, lpc, sub);
    else acc = satd_strips<S, 1>(src, wr, tw, th, p1, p2, stride, lpc, sub);
  }
  return group_sum(acc, lpc, sub, lane);
}

// The source block into shared memory as words.
template <class S>
__device__ __forceinline__ void stage_src(uint32_t* dst, const S* org, int stride, int w, int h, int lane) {
  constexpr int SPW = 4 / sizeof(S);
  const int wr = w / SPW;
  __syncwarp();
  for (int i = lane; i < wr * h; i += 32) {
    int row = i / wr, wd = i - row * wr;
    dst[i] = ldw(org + (ptrdiff_t)row * stride + wd * SPW);
  }
  __syncwarp();
}

template <class S>
__device__ __forceinline__ const S* plane_at(const DevPlanes& p, int plane, int x, int y) {
  return (const S*)p.base + (int64_t)plane * p.plane_elems + p.origin + (int64_t)y * p.stride + x;
}

// ---- dataflow queue ---------------------------------------------------------

// A ring slot of the resident engine holds the lap tag of its index (1 to
// 65535, so that consecutive laps differ and a zeroed slot matches none),
// the frame's generation in its slot (low 16 bits), frame and task.
__device__ __forceinline__ uint32_t ring_lap(int ring_shift, unsigned long long idx) {
  return (uint32_t)((idx >> ring_shift) % 65535ull) + 1u;
}
__device__ __forceinline__ unsigned long long ring_entry(int ring_shift, unsigned long long idx, uint32_t gen, int f,
                                                         int t) {
  return (unsigned long long)ring_lap(ring_shift, idx) << 48 | (unsigned long long)(gen & 0xffffu) << 32 |
         ((uint32_t)f << 24) | (uint32_t)t;
}

// Push task `t` of frame `f` (one thread): its last dependency just
// finished. `big`: into the queue of the tasks a CTA runs; `gen`: the
// frame's generation (the engine's rings).
__device__ __forceinline__ void push_ready(const LaunchDesc& L, int f, int t, bool big = false, uint32_t gen = 0) {
  unsigned long long* const ready = big ? L.ready_big : L.ready;
  const unsigned long long idx = atomicAdd(big ? L.tail_big : L.tail, 1ull);
  if (L.ring_shift) {  // the engine's ring: the host keeps fewer tasks in flight than it has slots
    st_release64(ready + (idx & ((1ull << L.ring_shift) - 1ull)), ring_entry(L.ring_shift, idx, gen, f, t));
  } else if (idx < (unsigned long long)L.total)
    st_release64(ready + idx, ((unsigned long long)__ldg(L.epoch) << 32) | ((uint32_t)f << 24) | (uint32_t)t);
  else
    atomicOr(L.status, kStatusBadTask);
}

__device__ __forceinline__ bool group_task_of(const LaunchDesc& L, const FrameDesc& F, int t);

// A finished task's dependents, task `dtask` in each lane where `rel`
// (all lanes call): each decrement that reaches zero makes its task ready.
// Where the launch counts finished tasks, the warp keeps the first task made
// ready (lowest lane) to run next itself, saving the push, the pop and the
// hand-over to another warp, unless `cont` already holds one; the others are
// pushed. Returns `cont`, updated.
// Tasks a CTA runs go to their own queue; a warp keeps only a task of its
// own kind (`group`: the caller is a CTA).
__device__ __forceinline__ int release_lanes(const LaunchDesc& L, const FrameDesc& F, int f, bool rel, int dtask,
                                             int cont, int lane, bool group = false) {
  const bool ready = rel && dec_acq_rel(&F.pending[dtask]) == 1;
  const bool big = ready && group_task_of(L, F, dtask);
  const uint32_t m = __ballot_sync(kFull, ready && big == group);
  if (__ballot_sync(kFull, ready) == 0u) return cont;
  int keep = -1;
  if (m != 0u && cont < 0 && (L.done != nullptr || L.ring_shift)) {
    keep = __ffs(m) - 1;
    cont = (f << 24) | __shfl_sync(kFull, dtask, keep);
  }
  if (ready && lane != keep) push_ready(L, f, dtask, big, F.gen);
  return cont;
}

__device__ __forceinline__ void red_add64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// The row form: the published word of a task another row owns, waited for
// until it carries this search's tag (bounded: kSpinLimit polls, then the
// status word's timeout bit and a zero vector, so that a lost dependency
// ends the search with an error instead of hanging it). The caller has
// loaded the word once already (`w`), while it staged its source. The first
// polls follow one another (the upper row is usually a block ahead, so the
// word comes within a few round trips); later ones back off.
__device__ __noinline__ unsigned long long wait_word(const LaunchDesc& L, const unsigned long long* p, uint32_t tag,
                                                     unsigned long long w) {
  uint32_t ns = 32;
  for (uint32_t it = 0; (uint32_t)(w >> 32) != tag; ++it) {
    if (it >= kSpinLimit) {
      atomicOr(L.status, kStatusWaitTimeout);
      return (unsigned long long)tag << 32;
    }
    if (it >= 16) {
      __nanosleep(ns);
      if (ns < 256) ns <<= 1;
    }
    w = ld_relaxed64(p);
  }
  return w;
}
__device__ __forceinline__ unsigned long long mv_word(uint32_t tag, int mvx, int mvy) {
  return (unsigned long long)tag << 32 | (uint32_t)(uint16_t)(int16_t)mvx | (uint32_t)(uint16_t)(int16_t)mvy << 16;
}

constexpr uint32_t kPopDone = 0xfffffffeu;  // every task of the launch is done

// The entry in slot `idx` once pushed (lane 0; bounded wait with backoff),
// kPopDone once every task is done (a slot that will never be filled: the
// warps that ran tasks they made ready pushed fewer than `total`), or
// 0xffffffff when the wait runs out (status set).
__device__ __forceinline__ uint32_t pop_slot(const LaunchDesc& L, unsigned long long idx, uint32_t epoch,
                                             bool big = false) {
  uint32_t ns = 32, it = 0;
  for (;;) {
    const unsigned long long v = ld_acquire64((big ? L.ready_big : L.ready) + idx);
    if ((uint32_t)(v >> 32) == epoch) return (uint32_t)v;
    if (L.done != nullptr && (it & 3u) == 3u && ld_relaxed64(L.done) >= (unsigned long long)L.total) return kPopDone;
    if (++it >= kSpinLimit) {
      atomicOr(L.status, kStatusWaitTimeout);
      return 0xffffffffu;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
}

__device__ __forceinline__ uint32_t ldcg_u32(const void* p) { return __ldcg((const unsigned int*)p); }
__device__ __forceinline__ int mvx_of(uint32_t v) { return (int)(int16_t)(v & 0xffffu); }
__device__ __forceinline__ int mvy_of(uint32_t v) { return (int)(int16_t)(v >> 16); }

// Per-warp totals of the work done, kept in shared memory (not registers)
// and added to the launch's counters once at exit.
template <class S>
__device__ __forceinline__ void count_task(WarpSmem<S>& sm, int lane, uint32_t nsad, uint32_t nsatd, int area) {
  if (lane == 0) {
    sm.cnt[0] += 1;
    sm.cnt[1] += nsad;
    sm.cnt[2] += nsatd;
    sm.cnt[3] += (unsigned long long)nsad * area;
    sm.cnt[4] += (unsigned long long)nsatd * area;
  }
}

// A GIVEN job as the host checks it before a launch (reference index,
// seed count, a block of 4..64 in multiples of 4 inside the coded picture).
// The kernel checks it again before reading anything the job points at,
// because jobs handed over in device memory never pass the host's check: a
// job that fails sets kStatusBadTask (the call returns RME_EDEVICE) and its
// result is left unwritten.
__device__ __forceinline__ bool given_job_ok(const FrameDesc& F, const rme_job* j, int max_seeds) {
  const int ref = j->ref, ns = j->nseeds, x = j->x, y = j->y, w = j->w, h = j->h;
  return ref >= 0 && ref < F.nref && ref < RME_MAX_REFS && ns >= 0 && ns <= max_seeds && w >= 4 && h >= 4 &&
         w <= 64 && h <= 64 && (w & 3) == 0 && (h & 3) == 0 && x >= 0 && y >= 0 && x <= F.width - w &&
         y <= F.height - h;
}

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
// (lam * mv_bits as f32) as u32 (h265_me.rs:3776, 3890): one IEEE
// round-to-nearest multiply, truncated.
__device__ __forceinline__ uint32_t hevc_rate(float lam, int mx, int my, int p0x, int p0y, int p1x, int p1y) {
  uint32_t b0 = hevc_cbits(mx - p0x) + hevc_cbits(my - p0y);
  uint32_t b1 = hevc_cbits(mx - p1x) + hevc_cbits(my - p1y);
  return __float2uint_rz(__fmul_rn(lam, __uint2float_rn(min(b0, b1) + 1u)));
}

// ---- HEVC scoring: one lane's part of a candidate ----------------------------
//
// A candidate is scored by a group of lanes. For SAD the group is eight
// lanes and lane `sub` sums rows sub, sub + 8, ...; square blocks of the
// STANDALONE sizes have their shape fixed at compile time (every load of a
// row issued before any is used, no division between a step's loads and
// its decision), other shapes go a word at a time.

template <class S, int WR, int RPL>
__device__ __forceinline__ uint32_t sad_rows_fixed(const uint32_t* src, const S* rp, int stride, int sub) {
  constexpr int SPW = 4 / sizeof(S), CW = WR < 8 ? WR : 8, UNR = RPL < 2 ? RPL : 2;
  uint32_t acc = 0;
#pragma unroll UNR
  for (int k = 0; k < RPL; ++k) {
    const int row = sub + 8 * k;
    const S* rr = rp + (ptrdiff_t)row * stride;
    const uint32_t* sr = src + row * WR;
#pragma unroll
    for (int c = 0; c < WR; c += CW) {
      uint32_t a[CW];
      ldwords<CW>(rr + c * SPW, a);
#pragma unroll
      for (int j = 0; j < CW; ++j) acc += vsad(sr[c + j], a[j], S());
    }
  }
  return acc;
}

template <class S>
__device__ __forceinline__ uint32_t sad_part(const uint32_t* src, int w, int h, const S* rp, int stride, int sub) {
  constexpr int SPW = 4 / sizeof(S);
  if (w == h) {
    if (w == 8) return sad_rows_fixed<S, 8 / SPW, 1>(src, rp, stride, sub);
    if (w == 16) return sad_rows_fixed<S, 16 / SPW, 2>(src, rp, stride, sub);
    if (w == 32) return sad_rows_fixed<S, 32 / SPW, 4>(src, rp, stride, sub);
    if (w == 64) return sad_rows_fixed<S, 64 / SPW, 8>(src, rp, stride, sub);
  }
  const int wr = w / SPW;
  uint32_t acc = 0;
  for (int row = sub; row < h; row += 8)
    for (int k = 0; k < wr; ++k) acc += vsad(src[row * wr + k], ldw(rp + (ptrdiff_t)row * stride + k * SPW), S());
  return acc;
}

// A 16x16 candidate's SAD over two lanes: rows half * 8 .. half * 8 + 7,
// loaded four rows at a time.
template <class S>
__device__ __forceinline__ uint32_t sad16_half(const uint32_t* src, const S* rp, int stride, int half) {
  constexpr int SPW = 4 / sizeof(S), WR = 16 / SPW;
  uint32_t acc = 0;
#pragma unroll
  for (int r0 = 0; r0 < 8; r0 += 4) {
    uint32_t a[4][WR];
#pragma unroll
    for (int r = 0; r < 4; ++r) ldwords<WR>(rp + (ptrdiff_t)(half * 8 + r0 + r) * stride, a[r]);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int k = 0; k < WR; ++k) acc += vsad(src[(half * 8 + r0 + r) * WR + k], a[r][k], S());
  }
  return acc;
}

// An 8x8 candidate's SAD over two lanes: rows half * 4 .. half * 4 + 3.
template <class S>
__device__ __forceinline__ uint32_t sad8_half(const uint32_t* src, const S* rp, int stride, int half) {
  constexpr int SPW = 4 / sizeof(S), WR = 8 / SPW;
  uint32_t a[4][WR];
#pragma unroll
  for (int r = 0; r < 4; ++r) ldwords<WR>(rp + (ptrdiff_t)(half * 4 + r) * stride, a[r]);
  uint32_t acc = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = 0; k < WR; ++k) acc += vsad(src[(half * 4 + r) * WR + k], a[r][k], S());
  return acc;
}

// SATD: lane `sub` of a group of G lanes takes the 4x4 tiles sub, sub + G,
// ... (row-major over tw tiles per row) of the candidate whose prediction
// starts at `pp`; each tile is the Hadamard of dsp/distortion.rs:326-381.
template <class S>
__device__ __forceinline__ uint32_t satd_part(const uint32_t* src, int wr, int tw, int ntiles, const S* pp, int stride,
                                              int sub, int G) {
  constexpr int SPW = 4 / sizeof(S), WPT = 4 / SPW;  // words per tile row
  const bool pow2 = (tw & (tw - 1)) == 0;
  const int sh = __ffs(tw) - 1;
  uint32_t acc = 0;
#pragma unroll 2
  for (int t = sub; t < ntiles; t += G) {
    const int ty = pow2 ? t >> sh : t / tw, tx = t - ty * tw;
    uint32_t pw[4][WPT];
#pragma unroll
    for (int r = 0; r < 4; ++r) ldwords<WPT>(pp + (ptrdiff_t)(ty * 4 + r) * stride + tx * 4, pw[r]);
    int d[16];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint32_t* srow = &src[(ty * 4 + r) * wr + tx * WPT];
#pragma unroll
      for (int k = 0; k < WPT; ++k) {
        const uint32_t sw = srow[k], qw = pw[r][k];
#pragma unroll
        for (int e = 0; e < SPW; ++e) {
          const int shf = e * (32 / SPW);
          const uint32_t m = SPW == 4 ? 0xffu : 0xffffu;
          d[r * 4 + k * SPW + e] = (int)((sw >> shf) & m) - (int)((qw >> shf) & m);
        }
      }
    }
    acc += satd4x4(d);
  }
  return acc;
}

// ---- 8x8 sub-sample refinement from staged phase patches (latency form) ----
//
// refine_subpel around a whole-sample best B only ever reads quarter-sample
// positions B + (qx, qy) with qx, qy in -3..3 (the half ring at +-2, then the
// quarter ring around its winner). Position B + q lies in phase plane
// ((qy & 3) * 4 + (qx & 3)) at whole-sample offset (floor(qx / 4),
// floor(qy / 4)), so every candidate's 8x8 prediction sits inside the 9x9
// block at B - (1, 1) of one of the 16 planes. Those 16 patches are staged
// in shared memory with one round of loads, and the reference's walk
// (start and half ring, then the quarter ring around the winner; strict <)
// scores its candidates from there: three dependent passes over the caches
// become one round of loads.
constexpr int kPatch = 9;        // patch rows and samples per row
constexpr int kPatchOff = 64;    // words of WarpSmem::src before the patches
template <class S>
struct PatchGeo {
  static constexpr int WR = sizeof(S) == 1 ? 3 : 5;  // words per staged row (any sample offset)
  static constexpr int PW = kPatch * WR;             // words per plane
  static constexpr int N = 16 * PW, PER = (N + 31) / 32;  // words staged, per lane
};
static_assert(kPatchOff + 16 * PatchGeo<uint16_t>::PW + 1 <= kMaxBlk * kMaxBlk / 2, "patches outgrew the source buffer");

// Stage the 16 planes' 9x9 patches at plane position (px, py) of R: word
// loads from the aligned word holding each row's first sample (all loads of
// a lane issued before any store); returns the byte offset of the first
// sample within its word (the same in every plane and row: planes and rows
// are whole words apart, which the caller checks).
template <class S>
__device__ __forceinline__ uint32_t load_patches(uint32_t (&v)[PatchGeo<S>::PER], const DevPlanes& R, int px, int py,
                                                 int lane) {
  using G = PatchGeo<S>;
  const S* p0 = (const S*)R.base + R.origin + (int64_t)py * R.stride + px;
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(p0);
  const uint32_t* w0 = reinterpret_cast<const uint32_t*>(a0 & ~uintptr_t(3));
  const int64_t pstep = R.plane_elems * (int64_t)sizeof(S) / 4, rstep = (int64_t)R.stride * sizeof(S) / 4;
#pragma unroll
  for (int k = 0; k < G::PER; ++k) {
    const int i = lane + 32 * k;
    v[k] = 0u;
    if (i < G::N) {
      const int pl = i / G::PW, rem = i - pl * G::PW, row = rem / G::WR, wd = rem - row * G::WR;
      v[k] = RME_LD32(w0 + pl * pstep + row * rstep + wd);
    }
  }
  return (uint32_t)(a0 & 3);
}
template <class S>
__device__ __forceinline__ void store_patches(uint32_t* dst, const uint32_t (&v)[PatchGeo<S>::PER], int lane) {
  using G = PatchGeo<S>;
#pragma unroll
  for (int k = 0; k < G::PER; ++k)
    if (lane + 32 * k < G::N) dst[lane + 32 * k] = v[k];
}
template <class S>
__device__ __forceinline__ uint32_t stage_patches(uint32_t* dst, const DevPlanes& R, int px, int py, int lane) {
  uint32_t v[PatchGeo<S>::PER];
  const uint32_t off = load_patches<S>(v, R, px, py, lane);
  store_patches<S>(dst, v, lane);
  return off;
}

// One 4x4 tile's SATD against the patch: tile (tx, ty) of the candidate
// whose 8x8 prediction starts at row sy, sample sx of patch `pp`.
template <class S>
__device__ __forceinline__ uint32_t patch_tile_satd(const uint32_t* src, const uint32_t* pp, uint32_t off, int sx,
                                                    int sy, int tx, int ty) {
  using G = PatchGeo<S>;
  constexpr int SPW = 4 / sizeof(S), WPT = 4 / SPW, SWR = 8 / SPW;
  int d[16];
  const uint32_t bit0 = (off + (uint32_t)((sx + tx * 4) * sizeof(S))) * 8u;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const uint32_t* prow = pp + (sy + ty * 4 + r) * G::WR;
    const uint32_t* srow = src + (ty * 4 + r) * SWR + tx * WPT;
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
      const uint32_t b = bit0 + 32u * k, wi = b >> 5, sh = b & 31u;
      const uint32_t qw = __funnelshift_r(prow[wi], prow[wi + 1], sh), sw = srow[k];
#pragma unroll
      for (int e = 0; e < SPW; ++e) {
        const int shf = e * (32 / SPW);
        const uint32_t m = SPW == 4 ? 0xffu : 0xffffu;
        d[r * 4 + k * SPW + e] = (int)((sw >> shf) & m) - (int)((qw >> shf) & m);
      }
    }
  }
  return satd4x4(d);
}

// refine_subpel of an 8x8 block around whole-sample (bx, by) from staged
// patches: the vector, its cost and SATD. The half step and then the
// quarter ring around its winner, both read from shared memory: one round
// of loads for the whole refinement.
template <class S>
__device__ __forceinline__ void refine8_patched(WarpSmem<S>& sm, const DevPlanes& R, int x, int y, int bx, int by,
                                                float lam, int p0x, int p0y, int p1x, int p1y, int quarter_cross,
                                                int lane, int& bmx, int& bmy, uint32_t& bc, uint32_t& bsatd,
                                                uint32_t& nsatd) {
  using G = PatchGeo<S>;
  uint32_t* patch = sm.src + kPatchOff;
  const uint32_t off = stage_patches<S>(patch, R, x + bx - 1, y + by - 1, lane);
  __syncwarp();
  const int imx = bx * 4, imy = by * 4;
  // The start and the half ring (lane 0 the start, lanes 1..8 the ring in
  // the reference's order: dy outer, dx inner, centre skipped), four lanes
  // per position (one 4x4 tile each), from the patches.
  auto score = [&](int c, int qx, int qy, int t) -> uint32_t {
    const int pl = (qy & 3) * 4 + (qx & 3);
    (void)c;
    return patch_tile_satd<S>(sm.src, patch + pl * G::PW, off, qx < 0 ? 0 : 1, qy < 0 ? 0 : 1, t & 1, t >> 1);
  };
  uint32_t sv = 0;
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int c = it * 8 + (lane >> 2);
    uint32_t v = 0;
    if (c < 9) {
      const int q = c == 0 ? 4 : (c <= 4 ? c - 1 : c);
      v = score(c, (q % 3 - 1) * 2, (q / 3 - 1) * 2, lane & 3);
    }
    v += __shfl_xor_sync(kFull, v, 1);
    v += __shfl_xor_sync(kFull, v, 2);
    const uint32_t got = __shfl_sync(kFull, v, ((lane - it * 8) & 7) * 4);
    if (lane >= it * 8 && lane < it * 8 + 8 && lane < 9) sv = got;
  }
  int mx = imx, my = imy;
  uint32_t cost = kInf;
  if (lane < 9) {
    const int q = lane == 0 ? 4 : (lane <= 4 ? lane - 1 : lane);
    mx = imx + (q % 3 - 1) * 2;
    my = imy + (q / 3 - 1) * 2;
    cost = sv + hevc_rate(lam, mx, my, p0x, p0y, p1x, p1y);
  }
  Pick p = warp_min(cost);
  bc = p.cost;
  bsatd = __shfl_sync(kFull, sv, p.lane);
  bmx = __shfl_sync(kFull, mx, p.lane);
  bmy = __shfl_sync(kFull, my, p.lane);
  // The quarter ring around the winner (the cross only when asked), from
  // the same patches: eight positions, four lanes each.
  const int hx = bmx - imx, hy = bmy - imy;
  const int c = lane >> 2, q = c < 4 ? c : c + 1, dx = q % 3 - 1, dy = q / 3 - 1;
  const bool ok = !(quarter_cross != 0 && dx != 0 && dy != 0);
  uint32_t v = ok ? score(c, hx + dx, hy + dy, lane & 3) : 0u;
  v += __shfl_xor_sync(kFull, v, 1);
  v += __shfl_xor_sync(kFull, v, 2);
  mx = (int)(int16_t)(bmx + dx);
  my = (int)(int16_t)(bmy + dy);
  cost = ok ? v + hevc_rate(lam, mx, my, p0x, p0y, p1x, p1y) : kInf;
  nsatd += 9 + __popc(__ballot_sync(kFull, ok && (lane & 3) == 0));
  p = warp_min(cost);
  if (p.cost < bc) {
    bc = p.cost;
    bsatd = __shfl_sync(kFull, v, p.lane);
    bmx = __shfl_sync(kFull, mx, p.lane);
    bmy = __shfl_sync(kFull, my, p.lane);
  }
}

// The row form's place in its row: level, block, reference.
struct RowPos {
  int l, lbx, lby, r;
};

__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Returns a task it made ready to run next (frame << 24 | task), or -1.
// SPEC: the latency kernels' two-rounds-per-step 8x8 and 16x16 diamond.
// ROW: the row form (the neighbours' vectors from their published words,
// this task's published in turn; nothing released), at `rp` in its row,
// blocks of NB samples (0: the level's size read at run time).
template <class S, bool SPEC, bool ROW = false, int NB = 0>
__device__ int hevc_task(const LaunchDesc& L, const FrameDesc& F, int f, int t, WarpSmem<S>& sm, int lane,
                         RowPos* rp = nullptr) {
  int r, x, y, w, h, ns;
  int p0x, p0y, p1x, p1y;
  int sx = 0, sy = 0;  // this lane's seed (lane < ns)
  int l = 0, lbx = 0, lby = 0, local = 0;  // STANDALONE: level and block
  bool amp_unit = false;                   // STANDALONE: an AMP unit
  rme_result* out;
  if (!ROW && F.mode == RME_PRED_GIVEN) {
    const rme_job* j = &F.jobs[t];
    if (!given_job_ok(F, j, RME_MAX_SEEDS)) {
      if (lane == 0) atomicOr(L.status, kStatusBadTask);
      return -1;
    }
    r = j->ref;
    x = j->x;
    y = j->y;
    w = j->w;
    h = j->h;
    ns = j->nseeds;
    p0x = j->mvp[0].x;
    p0y = j->mvp[0].y;
    p1x = j->mvp[1].x;
    p1y = j->mvp[1].y;
    if (lane < ns) {
      sx = j->seeds[lane].x;
      sy = j->seeds[lane].y;
    }
    out = &F.out[t];
  } else if (ROW) {
    r = rp->r;
  } else {
    r = t % F.nref;
    const int blk = t / F.nref;
    amp_unit = blk >= F.base[F.nlevels];
  }
  if (!ROW && amp_unit) {
    // An AMP unit (after every 2Nx2N block): its level, CU, mode and part.
    // It is searched from its CU's own 2Nx2N result: AMVP pair [own, 0],
    // seeds [own, mvp0, mvp1] (the parts search's own seed first).
    const int blk = t / F.nref;
    int la = 0;
    while (la + 1 < F.amp_nlev && blk >= F.amp_base[la + 1]) ++la;
    const int per = 2 * F.amp_nmodes, j = blk - F.amp_base[la], cu = j / per, rem = j - cu * per;
    int mode = 0;
    for (int b = 0, k = rem >> 1; b < 4; ++b)
      if ((F.amp >> b) & 1) {
        if (k == 0) {
          mode = b;
          break;
        }
        --k;
      }
    const int part = rem & 1, N = F.size[la], q = N / 4;
    const int cby = cu / F.nbx[la], cbx = cu - cby * F.nbx[la];
    x = cbx * N;
    y = cby * N;
    w = h = N;
    if (mode < 2) {
      h = (part == (mode == 0)) ? 3 * q : q;
      if (part) y += mode == 0 ? q : 3 * q;
    } else {
      w = (part == (mode == 2)) ? 3 * q : q;
      if (part) x += mode == 2 ? q : 3 * q;
    }
    const uint32_t ov = ldcg_u32(&F.out[(F.base[la] + cu) * F.nref + r].mv);
    stage_src<S>(sm.src, plane_at<S>(F.src, 0, x, y), F.src.stride, w, h, lane);
    p0x = mvx_of(ov);
    p0y = mvy_of(ov);
    p1x = p1y = 0;
    ns = 3;
    sx = lane == 0 || lane == 1 ? p0x : 0;
    sy = lane == 0 || lane == 1 ? p0y : 0;
    out = &F.out[t];
  } else if (ROW || F.mode != RME_PRED_GIVEN) {
    if (ROW) {
      l = rp->l;
      lbx = rp->lbx;
      lby = rp->lby;
      local = lby * F.nbx[l] + lbx;
    } else {
      const int blk = t / F.nref;
      while (l + 1 < F.nlevels && blk >= F.base[l + 1]) ++l;
      local = blk - F.base[l];
      lby = local / F.nbx[l];
      lbx = local - lby * F.nbx[l];
    }
    const int nbx = F.nbx[l];
    const int N = NB ? NB : F.size[l];
    x = lbx * N;
    y = lby * N;
    w = h = N;
    // The AMVP pair from the left and upper results of this level, the
    // parent seed from the enclosing block one evaluated size up (all of
    // them finished: the task was queued after its last dependency). Lanes
    // 0, 1, 2 load them together.
    int didx = -1;
    if (lane == 0 && lbx > 0) didx = (F.base[l] + local - 1) * F.nref + r;
    if (lane == 1 && lby > 0) didx = (F.base[l] + local - nbx) * F.nref + r;
    if (lane == 2 && l > 0) {
      const int Np = F.size[l - 1], px = x / Np, py = y / Np;
      if (px < F.nbx[l - 1] && py < F.nby[l - 1]) didx = (F.base[l - 1] + py * F.nbx[l - 1] + px) * F.nref + r;
    }
    uint32_t dv = 0u;
    unsigned long long dw = 0ull;
    if (ROW) {
      if (didx >= 0) dw = ld_relaxed64(F.mvf + didx);
    } else {
      dv = didx >= 0 ? ldcg_u32(&F.out[didx].mv) : 0u;
    }
    // The source block is staged while those loads are in flight.
    stage_src<S>(sm.src, plane_at<S>(F.src, 0, x, y), F.src.stride, w, h, lane);
    if (ROW && didx >= 0) dv = (uint32_t)wait_word(L, F.mvf + didx, F.tag, dw);
    // The row form: the next block's source rows brought into L1 now.
    if (ROW && lbx + 1 < nbx && lane < N) prefetch_l1(plane_at<S>(F.src, 0, x + N, y + lane));
    const uint32_t have = __ballot_sync(kFull, didx >= 0);
    const uint32_t va = __shfl_sync(kFull, dv, 0), vb = __shfl_sync(kFull, dv, 1), vp = __shfl_sync(kFull, dv, 2);
    int na = 0, ax = 0, ay = 0, cx = 0, cy = 0;
    if (have & 1u) {
      ax = mvx_of(va);
      ay = mvy_of(va);
      na = 1;
    }
    if (have & 2u) {
      const int qx = mvx_of(vb), qy = mvy_of(vb);
      if (na == 0) {
        ax = qx;
        ay = qy;
        na = 1;
      } else if (qx != ax || qy != ay) {
        cx = qx;
        cy = qy;
        na = 2;
      }
    }
    p0x = na > 0 ? ax : 0;
    p0y = na > 0 ? ay : 0;
    p1x = na > 1 ? cx : 0;
    p1y = na > 1 ? cy : 0;
    ns = (have & 4u) ? 4 : 3;
    const int psx = mvx_of(vp), psy = mvy_of(vp);
    // seeds = [zero, mvp0, mvp1, parent] (h265_me.rs:1327-1348)
    sx = lane == 1 ? p0x : lane == 2 ? p1x : lane == 3 ? psx : 0;
    sy = lane == 1 ? p0y : lane == 2 ? p1y : lane == 3 ? psy : 0;
    out = &F.out[t];
  }
  const DevPlanes& R = F.ref[r];
  if (!ROW && F.mode == RME_PRED_GIVEN) {
    if (F.bi_src)  // refine_bi: the target block stands in for the source
      stage_src<S>(sm.src, (const S*)F.bi_src + (int64_t)t * (kBiBlock * kBiBlock), kBiBlock, w, h, lane);
    else
      stage_src<S>(sm.src, plane_at<S>(F.src, 0, x, y), F.src.stride, w, h, lane);
  }
  const S* org = plane_at<S>(R, 0, x, y);
  const int stride = R.stride;
  constexpr int SPW = 4 / sizeof(S);
  const int wr = w / SPW, tw = w >> 2, th = h >> 2;
  const int padm = F.pad - 4;  // h265_search.rs MARGIN
  const int lox = -padm - x, hix = F.width + padm - w - x, loy = -padm - y, hiy = F.height + padm - h - y;
  const float lam = F.bi_src ? 2.0f * F.lam : F.lam;  // refine_bi weighs the rate at 2 * lam
  uint32_t nsad = 0, nsatd = 0;

  // Seeds: >> 2, clamp_pos, dedupe (a seed equal to an earlier one is
  // skipped: `tried`, h265_me.rs:3785-3800), scored in order.
  const int qx = min(max(sx >> 2, lox), hix), qy = min(max(sy >> 2, loy), hiy);
  bool dup = false;
#pragma unroll
  for (int j = 0; j < RME_MAX_SEEDS; ++j) {
    const int ox = __shfl_sync(kFull, qx, j), oy = __shfl_sync(kFull, qy, j);
    dup |= j < lane && ox == qx && oy == qy;
  }
  const uint32_t keep = __ballot_sync(kFull, lane < ns && !dup);
  const int nk = __popc(keep);
  const bool kept = (keep >> lane) & 1u;
  const int rank = __popc(keep & ((1u << lane) - 1u));

  // search_full as one loop of steps, each scoring four candidates (eight
  // lanes each; group g = lane / 8): the seeds four at a time, then the
  // small diamond rounds from a fixed `from`, then (search_rings) the 24
  // ring points four at a time, a move restarting the diamond. One scoring
  // site keeps the kernel's code small.
  const int g = lane >> 3, sub = lane & 7;
  const int range = F.search_range;
  int bx = 0, by = 0, ox = 0, oy = 0, cxr = 0, cyr = 0;
  uint32_t bcost = kInf;
  int state = nk > 0 ? 0 : 1, c0 = 0, it = 0, rings = 0;
  bool moved = false;
  const bool spec = SPEC && w == h && (w == 8 || w == 16);
  for (;;) {
    if (state == 1 && it >= 2 * range) {  // the diamond has settled
      if (rings >= F.search_rings) break;
      ++rings;
      state = 2;
      c0 = 0;
      moved = false;
      cxr = bx;
      cyr = by;
    }
    if (spec && state == 1) {
      // 8x8 and 16x16 in a latency kernel: two diamond rounds per step, fewer
      // dependent steps on the frame's critical path for more loads per step
      // (the throughput kernels keep one round per step, and leave this code
      // out of their text).
      // Candidates 0..3 (two lanes each)
      // are the round around the best; 4..15 the next round's points for
      // each way the first can move — three new ones each, the fourth being
      // the best itself, whose cost is known and cannot win. The outcome
      // and the count are those of the two rounds taken one after another.
      const int q = lane >> 1, hf = lane & 1;
      const int j0 = q < 4 ? q : (q - 4) / 3, mm = (q - 4) % 3, m = mm + (mm >= (j0 ^ 1));
      int fx = bx + (j0 == 0 ? 1 : j0 == 1 ? -1 : 0), fy = by + (j0 == 2 ? 1 : j0 == 3 ? -1 : 0);
      if (q >= 4) {
        fx += m == 0 ? 1 : m == 1 ? -1 : 0;
        fy += m == 2 ? 1 : m == 3 ? -1 : 0;
      }
      const bool ok = abs(fx - ox) <= range && abs(fy - oy) <= range && fx >= lox && fx <= hix && fy >= loy &&
                      fy <= hiy;
      uint32_t part = 0u;
      if (ok)
        part = w == 8 ? sad8_half<S>(sm.src, org + (ptrdiff_t)fy * stride + fx, stride, hf)
                      : sad16_half<S>(sm.src, org + (ptrdiff_t)fy * stride + fx, stride, hf);
      part += __shfl_xor_sync(kFull, part, 1);
      const uint32_t cost = ok ? part + hevc_rate(lam, fx * 4, fy * 4, p0x, p0y, p1x, p1y) : kInf;
      nsad += __popc(__ballot_sync(kFull, ok && hf == 0 && q < 4));
      const Pick pa = warp_min(q < 4 ? cost : kInf);
      if (!(pa.cost < bcost)) {
        it = 2 * range;
        continue;
      }
      const int j = pa.lane >> 1;
      bcost = pa.cost;
      bx = __shfl_sync(kFull, fx, pa.lane);
      by = __shfl_sync(kFull, fy, pa.lane);
      if (++it >= 2 * range) continue;
      const bool inb = q >= 4 && j0 == j;
      nsad += 1u + __popc(__ballot_sync(kFull, inb && ok && hf == 0));
      const Pick pb = warp_min(inb ? cost : kInf);
      if (pb.cost < bcost) {
        bcost = pb.cost;
        bx = __shfl_sync(kFull, fx, pb.lane);
        by = __shfl_sync(kFull, fy, pb.lane);
        ++it;
      } else {
        it = 2 * range;
      }
      continue;
    }
    int fx, fy;
    bool ok;
    if (state == 0) {
      // Candidate c0 + g: the kept seed of that rank.
      const uint32_t m0 = __ballot_sync(kFull, kept && rank == c0), m1 = __ballot_sync(kFull, kept && rank == c0 + 1),
                     m2 = __ballot_sync(kFull, kept && rank == c0 + 2),
                     m3 = __ballot_sync(kFull, kept && rank == c0 + 3);
      const uint32_t m = g == 0 ? m0 : g == 1 ? m1 : g == 2 ? m2 : m3;
      ok = m != 0u;
      const int from = ok ? __ffs(m) - 1 : 0;
      fx = __shfl_sync(kFull, qx, from);
      fy = __shfl_sync(kFull, qy, from);
    } else {
      if (state == 1) {  // (1,0), (-1,0), (0,1), (0,-1)
        fx = bx + (g == 0 ? 1 : g == 1 ? -1 : 0);
        fy = by + (g == 2 ? 1 : g == 3 ? -1 : 0);
      } else {  // (r,0), (-r,0), (0,r), (0,-r), (r,r), (-r,r), (r,-r), (-r,-r) for r = 4, 8, 16
        const int c = c0 + g, rr = c < 8 ? 4 : c < 16 ? 8 : 16, k8 = c & 7;
        fx = cxr + ((k8 == 0 || k8 == 4 || k8 == 6) ? rr : (k8 == 1 || k8 == 5 || k8 == 7) ? -rr : 0);
        fy = cyr + ((k8 == 2 || k8 == 4 || k8 == 5) ? rr : (k8 == 3 || k8 == 6 || k8 == 7) ? -rr : 0);
      }
      ok = abs(fx - ox) <= range && abs(fy - oy) <= range && fx >= lox && fx <= hix && fy >= loy && fy <= hiy;
      nsad += __popc(__ballot_sync(kFull, ok && sub == 0));
    }
    uint32_t part = ok ? sad_part<S>(sm.src, w, h, org + (ptrdiff_t)fy * stride + fx, stride, sub) : 0u;
    part += __shfl_xor_sync(kFull, part, 4);
    part += __shfl_xor_sync(kFull, part, 2);
    part += __shfl_xor_sync(kFull, part, 1);
    const uint32_t cost = ok ? part + hevc_rate(lam, fx * 4, fy * 4, p0x, p0y, p1x, p1y) : kInf;
    const Pick p = warp_min(cost);
    const bool better = p.cost < bcost;
    if (better) {
      bcost = p.cost;
      bx = __shfl_sync(kFull, fx, p.lane);
      by = __shfl_sync(kFull, fy, p.lane);
    }
    if (state == 0) {
      c0 += 4;
      if (c0 >= nk) {  // the descent is confined to +-range of the best seed
        nsad += nk;
        ox = bx;
        oy = by;
        state = 1;
        it = 0;
      }
    } else if (state == 1) {
      it = better ? it + 1 : 2 * range;
    } else {
      moved |= better;
      c0 += 4;
      if (c0 >= 24) {
        if (!moved) break;
        state = 1;
        it = 0;
      }
    }
  }
  const uint32_t int_cost = bcost;
  const int imx = bx * 4, imy = by * 4;

  // refine_subpel: candidate 0 the start, 1..8 the half-sample ring (dy in
  // {-2,0,2} outer, dx inner, centre skipped), in one step; then the
  // quarter-sample ring around the winner (the cross only when asked).
  // Passes: candidates 0..7 of the half step (four lanes each), candidate 8
  // (all lanes), the quarter step's 8 (four lanes each); a later pass wins
  // only when strictly cheaper, as in the reference's in-order walk.
  int bmx = imx, bmy = imy;
  uint32_t bc = kInf, bsatd = 0;
  const int ntiles = tw * th;
  // Patches need every plane and row a whole number of words apart (true
  // of the library's pictures: 128-byte strides).
  if (spec && w == 8 && L.patch8 && ((R.stride * (int)sizeof(S)) & 3) == 0 &&
      ((R.plane_elems * (int64_t)sizeof(S)) & 3) == 0) {
    refine8_patched<S>(sm, R, x, y, bx, by, lam, p0x, p0y, p1x, p1y, F.quarter_cross, lane, bmx, bmy, bc, bsatd,
                       nsatd);
  } else {
  for (int pass = 0; pass < 3; ++pass) {
    const int G = pass == 1 ? 32 : 4, c = pass == 1 ? 8 : lane >> 2, gsub = pass == 1 ? lane : lane & 3;
    int mx, my;
    bool ok;
    if (pass < 2) {
      const int q = c == 0 ? 4 : (c <= 4 ? c - 1 : c);
      mx = imx + (q % 3 - 1) * 2;
      my = imy + (q / 3 - 1) * 2;
      ok = true;
    } else {
      const int q = c < 4 ? c : c + 1, dx = q % 3 - 1, dy = q / 3 - 1;
      mx = (int)(int16_t)(bmx + dx);
      my = (int)(int16_t)(bmy + dy);
      ok = !(F.quarter_cross != 0 && dx != 0 && dy != 0);
      nsatd += __popc(__ballot_sync(kFull, ok && gsub == 0));
    }
    const S* pp = plane_at<S>(R, (my & 3) * 4 + (mx & 3), x + (mx >> 2), y + (my >> 2));
    uint32_t part = ok ? satd_part<S>(sm.src, wr, tw, ntiles, pp, stride, gsub, G) : 0u;
    for (int o = G >> 1; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    const uint32_t cost = ok ? part + hevc_rate(lam, mx, my, p0x, p0y, p1x, p1y) : kInf;
    const Pick p = warp_min(cost);
    if (p.cost < bc) {
      bc = p.cost;
      bsatd = __shfl_sync(kFull, part, p.lane);
      bmx = __shfl_sync(kFull, mx, p.lane);
      bmy = __shfl_sync(kFull, my, p.lane);
    }
  }
  nsatd += 9;
  }
  write_result(out, bmx, bmy, r, bc, bsatd, imx, imy, int_cost, nsad, nsatd, lane);
  int cont = -1;
  if (ROW) {
    if (lane == 0) st_relaxed64(F.mvf + t, mv_word(F.tag, bmx, bmy));
  } else if (!ROW && F.mode != RME_PRED_GIVEN && !amp_unit) {
    // The tasks reading this result: right and lower neighbours of this
    // level, the blocks of the next evaluated size inside this one, this
    // CU's AMP units; each lane releases one of them. Lane 0's result is
    // ordered before the other lanes' accesses by the warp barrier, and each
    // release is an acquire-release atomic, cumulative over it: no separate
    // fence.
    __syncwarp();
    int ncx = 0, ncy = 0, cx0 = 0, cy0 = 0;
    if (l + 1 < F.nlevels) {
      const int N = F.size[l], M = F.size[l + 1];
      cx0 = lbx * N / M;
      cy0 = lby * N / M;
      ncx = max(0, min((lbx + 1) * N / M, F.nbx[l + 1]) - cx0);
      ncy = max(0, min((lby + 1) * N / M, F.nby[l + 1]) - cy0);
    }
    const int namp = l < F.amp_nlev ? 2 * F.amp_nmodes : 0, nch = ncx * ncy, ndep = 2 + nch + namp;
    for (int k0 = 0; k0 < ndep; k0 += 32) {
      const int k = k0 + lane;
      int dtask = -1;
      if (k >= ndep) {
      } else if (k == 0) {
        if (lbx + 1 < F.nbx[l]) dtask = (F.base[l] + local + 1) * F.nref + r;
      } else if (k == 1) {
        if (lby + 1 < F.nby[l]) dtask = (F.base[l] + local + F.nbx[l]) * F.nref + r;
      } else if (k < 2 + nch) {
        const int c = k - 2, cy = cy0 + c / ncx, cx = cx0 + c % ncx;
        dtask = (F.base[l + 1] + cy * F.nbx[l + 1] + cx) * F.nref + r;
      } else {
        dtask = (F.amp_base[l] + local * namp + (k - 2 - nch)) * F.nref + r;
      }
      cont = release_lanes(L, F, f, dtask >= 0, dtask, cont, lane);
    }
  }
  count_task(sm, lane, nsad, nsatd, w * h);
  return cont;
}

// ---- HEVC, large blocks: one CTA per task (latency form) ----------------------
//
// A 32x32 or 64x64 block's search is the longest dependent chain of a
// frame (its level's wavefront has few blocks in flight, each of 1-4 K
// samples per candidate), so in the latency form a whole CTA runs one: the
// 256 threads split every step's candidate rows (SAD, a lane per word of a
// row: coalesced) or 4x4 tiles (SATD), each warp's sum is added into the
// candidate's cost in shared memory, and after one barrier every thread
// reads the step's costs and takes the same decision. The steps are the
// single-warp search's (a diamond round a step: at these sizes the
// candidates' samples, not the dependent round trips, bound a step), with
// the 24 ring points together and the start with the half ring together.
// Each decision is the reference's in-order strict-< walk over the step's
// candidates, so the results and the candidate counts are the single-warp
// search's.
constexpr int kGroupThreads = kWarpsPerBlock * 32;

template <class S>
struct alignas(16) GroupSmem {
  unsigned long long cnt[6];
  // Per step, each candidate's distortion, summed by the warps' atomic adds.
  // Three buffers in turn: a step adds into one, clears the next (read two
  // steps ago, before the last barrier) and its decision reads the one it
  // filled after its barrier.
  uint32_t cost[3][32];
  uint32_t bc[8];        // broadcasts: predictor words, the popped entry
  uint32_t src[kMaxBlk * kMaxBlk * sizeof(S) / 4];
};

// True for the tasks a CTA runs (32x32 and 64x64 STANDALONE blocks) when
// the launch has CTAs for them.
__device__ __forceinline__ bool group_task_of(const LaunchDesc& L, const FrameDesc& F, int t) {
  return L.group_ctas > 0 && F.mode == RME_PRED_STANDALONE && F.codec == RME_CODEC_HEVC && t / F.nref < F.big_end;
}

// The SADs of `nc` candidates of an N x N block: pos(c, fx, fy) gives
// candidate c's whole-sample offset and whether it is scored. A warp takes
// 32 / WR rows of one candidate at a time, a lane a word of a row (loads
// coalesced along the row; the word after a lane's comes from its neighbour,
// the row's last lane loads it), four such passes' loads in flight; each
// warp's sum is added into cost[b][c].
template <class S, int N, class Pos>
__device__ __forceinline__ void cta_sad(GroupSmem<S>& gs, int b, const S* org, int stride, int nc, Pos pos, int tid) {
  constexpr int SPW = 4 / sizeof(S), WR = N / SPW, RPW = 32 / WR, K = 4, STEP = kWarpsPerBlock * RPW;
  const int lane = tid & 31, warp = tid >> 5, wd = lane % WR, rsub = lane / WR;
  if (tid < 32) gs.cost[(b + 1) % 3][tid] = 0u;
  const int rows = nc * N;
  for (int r0 = warp * RPW; r0 < rows; r0 += K * STEP) {
    uint32_t lo[K], hi[K], sh[K];
    int cc[K], rw[K];
    bool ok[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int rr = r0 + k * STEP + rsub;
      ok[k] = false;
      cc[k] = 0;
      rw[k] = 0;
      lo[k] = hi[k] = sh[k] = 0u;
      if (rr < rows) {  // uniform over the warp, as is the candidate
        const int c = rr / N;
        int fx, fy;
        cc[k] = c;
        rw[k] = rr - c * N;
        ok[k] = pos(c, fx, fy);
        if (ok[k]) {
          const uintptr_t a = reinterpret_cast<uintptr_t>(org + (ptrdiff_t)(fy + rw[k]) * stride + fx);
          const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
          sh[k] = (uint32_t)(a & 3) * 8u;
          lo[k] = RME_LD32(q + wd);
          if (wd == WR - 1) hi[k] = RME_LD32(q + WR);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint32_t nx = __shfl_down_sync(kFull, lo[k], 1);
      if (wd != WR - 1) hi[k] = nx;
      uint32_t acc = ok[k] ? vsad(gs.src[rw[k] * WR + wd], __funnelshift_r(lo[k], hi[k], sh[k]), S()) : 0u;
      acc = __reduce_add_sync(kFull, acc);
      if (lane == 0 && ok[k]) atomicAdd(&gs.cost[b][cc[k]], acc);
    }
  }
  __syncthreads();
}

// The diamond's window: the reference's integer plane around a staging
// centre (scx, scy) (whole-sample offsets from the block), kWinR samples
// beyond the block on every side, staged in shared memory behind the
// GroupSmem with coalesced word loads. A diamond round from any best within
// kWinR - 1 of the centre reads only the window, so a walk restages every
// few rounds instead of reading four candidates' rows through the caches
// every round.
constexpr int kWinR = 4;
template <class S, int N>
struct WinGeo {
  static constexpr int ROWS = N + 2 * kWinR;
  static constexpr int WRW = (N + 2 * kWinR) * (int)sizeof(S) / 4 + 1;  // words per staged row (any sample offset)
};
static_assert(sizeof(GroupSmem<uint8_t>) + WinGeo<uint8_t, 64>::ROWS * WinGeo<uint8_t, 64>::WRW * 4 <=
                  kWarpsPerBlock * sizeof(WarpSmem<uint8_t>),
              "the window outgrew the CTA's shared memory");
static_assert(sizeof(GroupSmem<uint16_t>) + WinGeo<uint16_t, 64>::ROWS * WinGeo<uint16_t, 64>::WRW * 4 <=
                  kWarpsPerBlock * sizeof(WarpSmem<uint16_t>),
              "the window outgrew the CTA's shared memory");

// Stage the window around (scx, scy); returns the byte offset of its first
// sample within the first word (the same on every row: rows are whole words
// apart). All threads call; ends with a barrier.
template <class S, int N>
__device__ __forceinline__ uint32_t stage_window(uint32_t* win, const S* org, int stride, int scx, int scy, int tid) {
  using W = WinGeo<S, N>;
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(org + (ptrdiff_t)(scy - kWinR) * stride + (scx - kWinR));
  const uint32_t* w0 = reinterpret_cast<const uint32_t*>(a0 & ~uintptr_t(3));
  const int rstep = stride * (int)sizeof(S) / 4;
  for (int i = tid; i < W::ROWS * W::WRW; i += kGroupThreads) {
    const int row = i / W::WRW, wd = i - row * W::WRW;
    win[i] = RME_LD32(w0 + (ptrdiff_t)row * rstep + wd);
  }
  __syncthreads();
  return (uint32_t)(a0 & 3);
}

// The SADs of `nc` candidates, all within kWinR of the window's centre, from
// the window (a lane per word of a candidate row, each thread's words of a
// candidate summed, each warp's sum added into cost[b][c]).
template <class S, int N, class Pos>
__device__ __forceinline__ void cta_sad_win(GroupSmem<S>& gs, int b, const uint32_t* win, uint32_t off0, int scx,
                                            int scy, int nc, Pos pos, int tid) {
  using W = WinGeo<S, N>;
  constexpr int SPW = 4 / sizeof(S), WR = N / SPW, JOBS = N * WR, PER = JOBS / kGroupThreads;
  if (tid < 32) gs.cost[(b + 1) % 3][tid] = 0u;
  for (int c = 0; c < nc; ++c) {
    int fx, fy;
    if (!pos(c, fx, fy)) continue;
    const uint32_t b0 = off0 + (uint32_t)((fx - scx + kWinR) * (int)sizeof(S));
    const int r0 = fy - scy + kWinR;
    uint32_t acc = 0;
#pragma unroll
    for (int m = 0; m < PER; ++m) {
      const int j = tid + m * kGroupThreads, row = j / WR, k = j - row * WR;
      const uint32_t bb = b0 + 4u * k, wi = bb >> 2, sh = (bb & 3u) * 8u;
      const uint32_t* wr = win + (r0 + row) * W::WRW;
      acc += vsad(gs.src[row * WR + k], __funnelshift_r(wr[wi], wr[wi + 1], sh), S());
    }
    acc = __reduce_add_sync(kFull, acc);
    if ((tid & 31) == 0) atomicAdd(&gs.cost[b][c], acc);
  }
  __syncthreads();
}

// The SATDs of `nc` candidates (quarter-sample vectors from pos), 4x4 tiles
// split over the CTA (a warp's lanes on adjacent tiles of a tile row:
// coalesced), each warp's sum added into cost[b][c].
template <class S, int N, class Pos>
__device__ __forceinline__ void cta_satd(GroupSmem<S>& gs, int b, const DevPlanes& R, int x, int y, int nc, Pos pos,
                                         int tid) {
  constexpr int SPW = 4 / sizeof(S), WPT = 4 / SPW, TW = N / 4, NT = TW * TW, WR = N / SPW;
  if (tid < 32) gs.cost[(b + 1) % 3][tid] = 0u;
  const int jobs = nc * NT;
#pragma unroll 3
  for (int j0 = 0; j0 < jobs; j0 += kGroupThreads) {
    const int j = j0 + tid;
    uint32_t acc = 0;
    int c = 0;
    bool ok = false;
    if (j < jobs) {
      c = j / NT;
      const int i = j - c * NT, ty = i / TW, tx = i - ty * TW;
      int mx, my;
      ok = pos(c, mx, my);
      if (ok) {
        const S* pp = plane_at<S>(R, (my & 3) * 4 + (mx & 3), x + (mx >> 2) + tx * 4, y + (my >> 2) + ty * 4);
        uint32_t pw[4][WPT];
#pragma unroll
        for (int r = 0; r < 4; ++r) ldwords<WPT>(pp + (ptrdiff_t)r * R.stride, pw[r]);
        int d[16];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const uint32_t* srow = &gs.src[(ty * 4 + r) * WR + tx * WPT];
#pragma unroll
          for (int k = 0; k < WPT; ++k) {
            const uint32_t sw = srow[k], qw = pw[r][k];
#pragma unroll
            for (int e = 0; e < SPW; ++e) {
              const int shf = e * (32 / SPW);
              const uint32_t m = SPW == 4 ? 0xffu : 0xffffu;
              d[r * 4 + k * SPW + e] = (int)((sw >> shf) & m) - (int)((qw >> shf) & m);
            }
          }
        }
        acc = satd4x4(d);
      }
    }
    acc = __reduce_add_sync(kFull, acc);  // a warp's 32 jobs are tiles of one candidate (NT >= 64)
    if ((tid & 31) == 0 && ok) atomicAdd(&gs.cost[b][c], acc);
  }
  __syncthreads();
}

// search_full + refine_subpel of one STANDALONE square block of N in {32, 64}
// by the whole CTA (all threads call). Returns a task it made ready to run
// next (frame << 24 | task; another group task) or -1.
template <class S, int N, bool ROW = false>
__device__ int hevc_group_task(const LaunchDesc& L, const FrameDesc& F, int f, int t, GroupSmem<S>& gs, int tid) {
  constexpr int SPW = 4 / sizeof(S), WR = N / SPW;
  const int lane = tid & 31;
  const int r = t % F.nref, blk = t / F.nref;
  int l = 0;
  while (l + 1 < F.nlevels && blk >= F.base[l + 1]) ++l;
  const int local = blk - F.base[l], nbx = F.nbx[l], lby = local / nbx, lbx = local - lby * nbx;
  const int x = lbx * N, y = lby * N;
  // The left, upper and parent results (threads 0..2), while all threads
  // stage the source block.
  int didx = -1;
  unsigned long long dw = 0ull;
  if (tid < 3) {
    if (tid == 0 && lbx > 0) didx = (F.base[l] + local - 1) * F.nref + r;
    if (tid == 1 && lby > 0) didx = (F.base[l] + local - nbx) * F.nref + r;
    if (tid == 2 && l > 0) {
      const int Np = F.size[l - 1], px = x / Np, py = y / Np;
      if (px < F.nbx[l - 1] && py < F.nby[l - 1]) didx = (F.base[l - 1] + py * F.nbx[l - 1] + px) * F.nref + r;
    }
    if (ROW) {
      if (didx >= 0) dw = ld_relaxed64(F.mvf + didx);
    } else {
      gs.bc[tid] = didx >= 0 ? ldcg_u32(&F.out[didx].mv) : 0u;
    }
    gs.bc[3 + tid] = didx >= 0 ? 1u : 0u;
  }
  if (tid < 64) gs.cost[tid >> 5][tid & 31] = 0u;  // the first step's buffer (and the next)
  {
    const S* so = plane_at<S>(F.src, 0, x, y);
    for (int i = tid; i < WR * N; i += kGroupThreads) {
      const int row = i / WR, wd = i - row * WR;
      gs.src[i] = ldw(so + (ptrdiff_t)row * F.src.stride + wd * SPW);
    }
  }
  if (ROW && tid < 3) gs.bc[tid] = didx >= 0 ? (uint32_t)wait_word(L, F.mvf + didx, F.tag, dw) : 0u;
  __syncthreads();
  int p0x = 0, p0y = 0, p1x = 0, p1y = 0, na = 0;
  if (gs.bc[3]) {
    p0x = mvx_of(gs.bc[0]);
    p0y = mvy_of(gs.bc[0]);
    na = 1;
  }
  if (gs.bc[4]) {
    const int qx = mvx_of(gs.bc[1]), qy = mvy_of(gs.bc[1]);
    if (na == 0) {
      p0x = qx;
      p0y = qy;
      na = 1;
    } else if (qx != p0x || qy != p0y) {
      p1x = qx;
      p1y = qy;
      na = 2;
    }
  }
  const int ns = gs.bc[5] ? 4 : 3;
  const int sdx[4] = {0, p0x, p1x, mvx_of(gs.bc[2])}, sdy[4] = {0, p0y, p1y, mvy_of(gs.bc[2])};
  const DevPlanes& R = F.ref[r];
  const S* org = plane_at<S>(R, 0, x, y);
  const int stride = R.stride;
  const int padm = F.pad - 4;  // h265_search.rs MARGIN
  const int lox = -padm - x, hix = F.width + padm - N - x, loy = -padm - y, hiy = F.height + padm - N - y;
  const float lam = F.lam;
  const int range = F.search_range;
  uint32_t nsad = 0, nsatd = 0;
  int buf = 0;  // the cost buffer of the next step (cta_sad / cta_satd)
  auto next = [&] { buf = buf == 2 ? 0 : buf + 1; };
  // Seeds: >> 2 (floor), clamp_pos, dedupe through `tried`, in order
  // (seed i is scored unless an earlier one landed on the same point).
  int kx[4], ky[4];
  bool kept[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    kx[i] = min(max(sdx[i] >> 2, lox), hix);
    ky[i] = min(max(sdy[i] >> 2, loy), hiy);
    bool dup = i >= ns;
#pragma unroll
    for (int j = 0; j < i; ++j) dup |= kx[j] == kx[i] && ky[j] == ky[i];
    kept[i] = !dup;
  }
  auto spos = [&](int c, int& fx, int& fy) {
    fx = c == 0 ? kx[0] : c == 1 ? kx[1] : c == 2 ? kx[2] : kx[3];
    fy = c == 0 ? ky[0] : c == 1 ? ky[1] : c == 2 ? ky[2] : ky[3];
    return c == 0 ? kept[0] : c == 1 ? kept[1] : c == 2 ? kept[2] : kept[3];
  };
  int bx = 0, by = 0;
  uint32_t bcost = kInf;
  cta_sad<S, N>(gs, buf, org, stride, 4, spos, tid);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int fx, fy;
    if (!spos(c, fx, fy)) continue;
    ++nsad;
    const uint32_t cost = gs.cost[buf][c] + hevc_rate(lam, fx * 4, fy * 4, p0x, p0y, p1x, p1y);
    if (cost < bcost) {
      bcost = cost;
      bx = fx;
      by = fy;
    }
  }
  next();
  const int ox = bx, oy = by;  // the descent stays within +-range of the best seed
  auto inside = [&](int fx, int fy) {
    return abs(fx - ox) <= range && abs(fy - oy) <= range && fx >= lox && fx <= hix && fy >= loy && fy <= hiy;
  };
  int rings = 0;
  uint32_t* const win = reinterpret_cast<uint32_t*>(&gs + 1);
  int scx = 0, scy = 0;
  uint32_t woff = 0;
  bool staged = false;
  for (;;) {
    // The small diamond, a round a step: (1,0), (-1,0), (0,1), (0,-1)
    // around the best, taken in order when strictly cheaper; scored from
    // the window, restaged around the best when the round would leave it.
    for (int it = 0; it < 2 * range; ++it) {
      const int cbx = bx, cby = by;
      auto pos = [&](int q, int& fx, int& fy) {
        fx = cbx + (q == 0 ? 1 : q == 1 ? -1 : 0);
        fy = cby + (q == 2 ? 1 : q == 3 ? -1 : 0);
        return inside(fx, fy);
      };
      if (!staged || abs(cbx - scx) > kWinR - 1 || abs(cby - scy) > kWinR - 1) {
        scx = cbx;
        scy = cby;
        woff = stage_window<S, N>(win, org, stride, scx, scy, tid);
        staged = true;
      }
      cta_sad_win<S, N>(gs, buf, win, woff, scx, scy, 4, pos, tid);
      bool improved = false;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int fx, fy;
        if (!pos(q, fx, fy)) continue;
        ++nsad;
        const uint32_t cost = gs.cost[buf][q] + hevc_rate(lam, fx * 4, fy * 4, p0x, p0y, p1x, p1y);
        if (cost < bcost) {
          bcost = cost;
          bx = fx;
          by = fy;
          improved = true;
        }
      }
      next();
      if (!improved) break;
    }
    if (rings >= F.search_rings) break;
    ++rings;
    // The 24 ring points at 4, 8, 16 around the settled point, together.
    const int cxr = bx, cyr = by;
    auto rpos = [&](int c, int& fx, int& fy) {
      const int rr = c < 8 ? 4 : c < 16 ? 8 : 16, k8 = c & 7;
      fx = cxr + ((k8 == 0 || k8 == 4 || k8 == 6) ? rr : (k8 == 1 || k8 == 5 || k8 == 7) ? -rr : 0);
      fy = cyr + ((k8 == 2 || k8 == 4 || k8 == 5) ? rr : (k8 == 3 || k8 == 6 || k8 == 7) ? -rr : 0);
      return inside(fx, fy);
    };
    cta_sad<S, N>(gs, buf, org, stride, 24, rpos, tid);
    bool moved = false;
    for (int c = 0; c < 24; ++c) {
      int fx, fy;
      if (!rpos(c, fx, fy)) continue;
      ++nsad;
      const uint32_t cost = gs.cost[buf][c] + hevc_rate(lam, fx * 4, fy * 4, p0x, p0y, p1x, p1y);
      if (cost < bcost) {
        bcost = cost;
        bx = fx;
        by = fy;
        moved = true;
      }
    }
    next();
    if (!moved) break;
  }
  const uint32_t int_cost = bcost;
  const int imx = bx * 4, imy = by * 4;
  // refine_subpel: the start and the half ring (dy outer, dx inner) in one
  // step, then the quarter ring around the winner.
  auto hpos = [&](int c, int& mx, int& my) {
    const int q = c == 0 ? 4 : (c <= 4 ? c - 1 : c);
    mx = imx + (q % 3 - 1) * 2;
    my = imy + (q / 3 - 1) * 2;
    return true;
  };
  cta_satd<S, N>(gs, buf, R, x, y, 9, hpos, tid);
  int bmx = imx, bmy = imy;
  uint32_t bc = kInf, bsatd = 0;
  for (int c = 0; c < 9; ++c) {
    int mx, my;
    hpos(c, mx, my);
    const uint32_t sv = gs.cost[buf][c], cost = sv + hevc_rate(lam, mx, my, p0x, p0y, p1x, p1y);
    if (cost < bc) {
      bc = cost;
      bsatd = sv;
      bmx = mx;
      bmy = my;
    }
  }
  next();
  const int hmx = bmx, hmy = bmy, cross = F.quarter_cross;
  auto qpos = [&](int c, int& mx, int& my) {
    const int q = c < 4 ? c : c + 1, dx = q % 3 - 1, dy = q / 3 - 1;
    mx = (int)(int16_t)(hmx + dx);
    my = (int)(int16_t)(hmy + dy);
    return !(cross != 0 && dx != 0 && dy != 0);
  };
  cta_satd<S, N>(gs, buf, R, x, y, 8, qpos, tid);
  for (int c = 0; c < 8; ++c) {
    int mx, my;
    if (!qpos(c, mx, my)) continue;
    ++nsatd;
    const uint32_t sv = gs.cost[buf][c], cost = sv + hevc_rate(lam, mx, my, p0x, p0y, p1x, p1y);
    if (cost < bc) {
      bc = cost;
      bsatd = sv;
      bmx = mx;
      bmy = my;
    }
  }
  nsatd += 9;
  rme_result* out = &F.out[t];
  if (tid == 0) {
    write_result(out, bmx, bmy, r, bc, bsatd, imx, imy, int_cost, nsad, nsatd, 0);
    gs.cnt[0] += 1;
    gs.cnt[1] += nsad;
    gs.cnt[2] += nsatd;
    gs.cnt[3] += (unsigned long long)nsad * N * N;
    gs.cnt[4] += (unsigned long long)nsatd * N * N;
    if (ROW) st_relaxed64(F.mvf + t, mv_word(F.tag, bmx, bmy));
  }
  __syncthreads();
  if (ROW) return -1;
  // The tasks reading this result (warp 0 releases them, one per lane):
  // right and lower neighbours, the next size's blocks inside this one,
  // this CU's AMP units. A group task made ready is kept, if this CTA has
  // none yet; the rest are pushed to their queues.
  int cont = -1;
  if (tid < 32) {
    int ncx = 0, ncy = 0, cx0 = 0, cy0 = 0;
    if (l + 1 < F.nlevels) {
      const int M = F.size[l + 1];
      cx0 = lbx * N / M;
      cy0 = lby * N / M;
      ncx = max(0, min((lbx + 1) * N / M, F.nbx[l + 1]) - cx0);
      ncy = max(0, min((lby + 1) * N / M, F.nby[l + 1]) - cy0);
    }
    const int namp = l < F.amp_nlev ? 2 * F.amp_nmodes : 0, nch = ncx * ncy, ndep = 2 + nch + namp;
    for (int k0 = 0; k0 < ndep; k0 += 32) {
      const int k = k0 + lane;
      int dtask = -1;
      if (k >= ndep) {
      } else if (k == 0) {
        if (lbx + 1 < F.nbx[l]) dtask = (F.base[l] + local + 1) * F.nref + r;
      } else if (k == 1) {
        if (lby + 1 < F.nby[l]) dtask = (F.base[l] + local + F.nbx[l]) * F.nref + r;
      } else if (k < 2 + nch) {
        const int c = k - 2, cy = cy0 + c / ncx, cx = cx0 + c % ncx;
        dtask = (F.base[l + 1] + cy * F.nbx[l + 1] + cx) * F.nref + r;
      } else {
        dtask = (F.amp_base[l] + local * namp + (k - 2 - nch)) * F.nref + r;
      }
      cont = release_lanes(L, F, f, dtask >= 0, dtask, cont, lane, true);
    }
    if (tid == 0) gs.bc[6] = (uint32_t)cont;
  }
  __syncthreads();
  return (int)gs.bc[6];
}

// ---- the row form ------------------------------------------------------------

// One row of an HEVC STANDALONE frame (a row_entry), its blocks left to right
// by this warp (8x8 and 16x16) or this CTA (32x32 and 64x64). A block waits
// only for the published vectors of its upper neighbour (the row above,
// which its owner started earlier and runs ahead of this one) and of its
// parent one size up; its left neighbour is this row's previous block. No
// dependency counts, no queue traffic between the blocks of a row.
__device__ __forceinline__ bool row_ok(const FrameDesc& F, uint32_t e, int& l, int& r, int& row) {
  l = (int)((e >> 22) & 3u);
  r = (int)((e >> 20) & 3u);
  row = (int)(e & 0xfffffu);
  return F.mvf != nullptr && F.codec == RME_CODEC_HEVC && F.mode == RME_PRED_STANDALONE && F.amp == 0 &&
         l < F.nlevels && r < F.nref && row < F.nby[l];
}

template <class S, bool SPEC>
__device__ void hevc_row(const LaunchDesc& L, const FrameDesc& F, int f, uint32_t e, WarpSmem<S>& sm, int lane) {
  int l, r, row;
  if (!row_ok(F, e, l, r, row) || (F.size[l] != 8 && F.size[l] != 16)) {
    if (lane == 0) atomicOr(L.status, kStatusBadTask);
    return;
  }
  const int nbx = F.nbx[l], t0 = (F.base[l] + row * nbx) * F.nref + r;
  RowPos rp{l, 0, row, r};
  if (F.size[l] == 8)
    for (int bx = 0; bx < nbx; ++bx) {
      rp.lbx = bx;
      hevc_task<S, SPEC, true, 8>(L, F, f, t0 + bx * F.nref, sm, lane, &rp);
    }
  else
    for (int bx = 0; bx < nbx; ++bx) {
      rp.lbx = bx;
      hevc_task<S, SPEC, true, 16>(L, F, f, t0 + bx * F.nref, sm, lane, &rp);
    }
}

template <class S>
__device__ void hevc_group_row(const LaunchDesc& L, const FrameDesc& F, int f, uint32_t e, GroupSmem<S>& gs,
                               int tid) {
  int l, r, row;
  if (!row_ok(F, e, l, r, row) || (F.size[l] != 32 && F.size[l] != 64)) {
    if (tid == 0) atomicOr(L.status, kStatusBadTask);
    return;
  }
  const int nbx = F.nbx[l], t0 = (F.base[l] + row * nbx) * F.nref + r;
  if (F.size[l] == 64)
    for (int bx = 0; bx < nbx; ++bx) hevc_group_task<S, 64, true>(L, F, f, t0 + bx * F.nref, gs, tid);
  else
    for (int bx = 0; bx < nbx; ++bx) hevc_group_task<S, 32, true>(L, F, f, t0 + bx * F.nref, gs, tid);
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
  int px, py;          // predictor (quarter samples)
  int lx, hx, ly, hy;  // search_bounds
  int wr, ipc, tw, th, tpc;
};

__device__ __forceinline__ uint32_t h264_rate(const FrameDesc& F, const H264Blk& B, int qx, int qy) {
  const int dx = min(max(qx - B.px, -kMvSpan), kMvSpan), dy = min(max(qy - B.py, -kMvSpan), kMvSpan);
  return (uint32_t)__ldg(&F.tab[dx + kMvSpan]) + (uint32_t)__ldg(&F.tab[dy + kMvSpan]);
}

// ring(): up to n points around a fixed centre (candidate c at offset
// off(c)), those inside the box and not the centre, scored in one step;
// returns the index of the point taken, or -1.
template <class S, class Off>
__device__ __forceinline__ int h264_ring(const FrameDesc& F, const H264Blk& B, WarpSmem<S>& sm, const S* org,
                                         int stride, int lane, int n, Off off, const int box[4], int& bx, int& by,
                                         uint32_t& bcost, uint32_t& nsad) {
  const int cx = bx, cy = by;
  const int lpc = lanes_per(n), cpp = 32 / lpc, sub = lane % lpc;
  int moved = -1;
  for (int c0 = 0; c0 < n; c0 += cpp) {
    const int c = lane / lpc < cpp ? c0 + lane / lpc : n;
    int ox = 0, oy = 0;
    off(c < n ? c : 0, ox, oy);
    const int fx = cx + ox, fy = cy + oy;
    const bool ok = c < n && fx >= box[0] && fx <= box[1] && fy >= box[2] && fy <= box[3] && !(fx == cx && fy == cy);
    const uint32_t s = group_sad<S>(sm.src, B.wr, B.h, org, stride, lpc, sub, lane, ok, fx, fy);
    const uint32_t cost = ok ? s + h264_rate(F, B, fx * 4, fy * 4) : kInf;
    nsad += __popc(__ballot_sync(kFull, ok && sub == 0));
    const Pick p = warp_min(cost);
    if (p.cost < bcost) {
      bcost = p.cost;
      bx = __shfl_sync(kFull, fx, p.lane);
      by = __shfl_sync(kFull, fy, p.lane);
      moved = __shfl_sync(kFull, c, p.lane);
    }
  }
  return moved;
}

// Search::int_search (h264_hpel.rs:789-952) for one reference: lane k + 1
// holds candidate k of `ncand` (quarter samples).
template <class S>
__device__ void h264_int_search(const FrameDesc& F, const H264Blk& B, WarpSmem<S>& sm, int lane, const DevPlanes& R,
                                int ncand, int cand_x, int cand_y, int& imx, int& imy, uint32_t& icost,
                                uint32_t& nsad) {
  const S* org = plane_at<S>(R, 0, B.x, B.y);
  const int stride = R.stride;
  // Candidate list: slot 0 the rounded, clamped predictor; slot k >= 1 the
  // candidate k-1, skipped when it equals the predictor's point or an
  // earlier candidate's (`tried`).
  const int pxr = min(max((B.px + 2) >> 2, B.lx), B.hx), pyr = min(max((B.py + 2) >> 2, B.ly), B.hy);
  const int cl = lane - 1;
  const int qx = lane == 0 ? pxr : min(max((cand_x + 2) >> 2, B.lx), B.hx);
  const int qy = lane == 0 ? pyr : min(max((cand_y + 2) >> 2, B.ly), B.hy);
  bool skip = lane > 0 && (qx == pxr && qy == pyr);
#pragma unroll
  for (int j = 1; j <= 8; ++j) {
    const int ox = __shfl_sync(kFull, qx, j), oy = __shfl_sync(kFull, qy, j);
    skip |= j < lane && ox == qx && oy == qy;
  }
  const uint32_t keep = __ballot_sync(kFull, (lane == 0 || cl < ncand) && !skip);
  const int nk = __popc(keep);
  int bx = pxr, by = pyr;
  uint32_t bcost = kInf;
  {
    const int lpc = lanes_per(nk), cpp = 32 / lpc, sub = lane % lpc;
    for (int c0 = 0; c0 < nk; c0 += cpp) {
      const int c = lane / lpc < cpp ? c0 + lane / lpc : nk;
      const bool ok = c < nk;
      const int from = ok ? __fns(keep, 0, c + 1) : 0;
      const int fx = __shfl_sync(kFull, qx, from), fy = __shfl_sync(kFull, qy, from);
      const uint32_t s = group_sad<S>(sm.src, B.wr, B.h, org, stride, lpc, sub, lane, ok, fx, fy);
      const uint32_t cost = ok ? s + h264_rate(F, B, fx * 4, fy * 4) : kInf;
      const Pick p = warp_min(cost);
      if (p.cost < bcost) {
        bcost = p.cost;
        bx = __shfl_sync(kFull, fx, p.lane);
        by = __shfl_sync(kFull, fy, p.lane);
      }
    }
  }
  nsad += nk;
  const int range = F.range;
  const int box[4] = {max(bx - range, B.lx), min(bx + range, B.hx), max(by - range, B.ly), min(by + range, B.hy)};
  if (F.umh) {
    // The cross r = 2, 4, .. range then 12-point hexagon rings r = 4, 8, ..
    // range around the fixed start, each point taken by try_at: skipped
    // (and not scored) when outside the box or equal to the best so far.
    const int cx = bx, cy = by;
    const int ncross = 4 * (range / 2), nhex = 12 * (range / 4), total = ncross + nhex;
    for (int c0 = 0; c0 < total; c0 += 32) {
      const int i = c0 + lane;
      int qx2 = 0, qy2 = 0;
      bool ok = i < total;
      if (ok) {
        if (i < ncross) {
          const int rr = 2 * (i / 4 + 1), k = i & 3;
          qx2 = cx + (k == 0 ? -rr : k == 1 ? rr : 0);
          qy2 = cy + (k == 2 ? -rr : k == 3 ? rr : 0);
        } else {
          const int j = i - ncross, rr = 4 * (j / 12 + 1), k = j % 12;
          qx2 = cx + c_hex12[k][0] * rr / 2;
          qy2 = cy + c_hex12[k][1] * rr / 2;
        }
        ok = qx2 >= box[0] && qx2 <= box[1] && qy2 >= box[2] && qy2 <= box[3];
      }
      const uint32_t s = group_sad<S>(sm.src, B.wr, B.h, org, stride, 1, 0, lane, ok, qx2, qy2);
      const uint32_t cost = ok ? s + h264_rate(F, B, qx2 * 4, qy2 * 4) : kInf;
      // In-order walk for the count of points scored (equal-to-best ones
      // are not); the outcome is the step's least cost, first reached.
      __syncwarp();
      sm.ux[lane] = qx2;
      sm.uy[lane] = qy2;
      sm.uc[lane] = ok ? cost : kInf;
      __syncwarp();
      int wx = bx, wy = by;
      uint32_t wc = bcost, scored = 0;
      const int np = min(32, total - c0);
      for (int k = 0; k < np; ++k) {
        const uint32_t ck = sm.uc[k];
        if (ck == kInf) continue;
        const int kx = sm.ux[k], ky = sm.uy[k];
        if (kx == wx && ky == wy) continue;
        ++scored;
        if (ck < wc) {
          wc = ck;
          wx = kx;
          wy = ky;
        }
      }
      nsad += scored;
      bx = wx;
      by = wy;
      bcost = wc;
    }
  }
  if (F.dia) {
    for (int it = 0; it < range; ++it) {
      const int cx = bx, cy = by;
      h264_ring<S>(F, B, sm, org, stride, lane, 4,
                   [](int c, int& ox, int& oy) {
                     ox = c == 0 ? -1 : c == 1 ? 1 : 0;
                     oy = c == 2 ? -1 : c == 3 ? 1 : 0;
                   },
                   box, bx, by, bcost, nsad);
      if (bx == cx && by == cy) break;
    }
  } else {
    int dir = h264_ring<S>(F, B, sm, org, stride, lane, 6,
                           [](int c, int& ox, int& oy) {
                             ox = c_hex[c][0];
                             oy = c_hex[c][1];
                           },
                           box, bx, by, bcost, nsad);
    int it = 1;
    while (dir != -1 && it < range) {
      const int d = dir;
      const int moved = h264_ring<S>(F, B, sm, org, stride, lane, 3,
                                     [d](int c, int& ox, int& oy) {
                                       const int k = c == 0 ? (d + 5) % 6 : c == 1 ? d : (d + 1) % 6;
                                       ox = c_hex[k][0];
                                       oy = c_hex[k][1];
                                     },
                                     box, bx, by, bcost, nsad);
      dir = moved == -1 ? -1 : (moved == 0 ? (d + 5) % 6 : moved == 1 ? d : (d + 1) % 6);
      ++it;
    }
    h264_ring<S>(F, B, sm, org, stride, lane, 8,
                 [](int c, int& ox, int& oy) {
                   ox = c_sq[c][0];
                   oy = c_sq[c][1];
                 },
                 box, bx, by, bcost, nsad);
  }
  imx = bx * 4;
  imy = by * 4;
  icost = bcost;
}

// Search::refine (h264_hpel.rs:956-1021) from (smx, smy): the start, then
// `hpel` rings of half-sample points and `qpel` of quarter-sample points
// (the start scored in the same step as the first ring).
template <class S>
__device__ void h264_refine(const FrameDesc& F, const H264Blk& B, WarpSmem<S>& sm, int lane, const DevPlanes& R, int smx,
                            int smy, int hpel, int qpel, int& omx, int& omy, uint32_t& osatd, uint32_t& ocost,
                            uint32_t& nsatd) {
  const int qlx = B.lx * 4, qhx = B.hx * 4, qly = B.ly * 4, qhy = B.hy * 4;
  int bmx = smx, bmy = smy;
  uint32_t bsatd = 0, bc = kInf;
  bool first = true;
  for (int s = 0; s < 2; ++s) {
    const int step = s == 0 ? 2 : 1, iters = s == 0 ? hpel : qpel;
    const int pts = (step == 1 && F.qpel_diamond) ? 4 : 8;
    bool has_prev = false;
    int prevx = 0, prevy = 0;
    for (int it = 0; it < iters || first; ++it) {
      const int cmx = bmx, cmy = bmy;
      const bool ring = it < iters;
      // Candidate 0 the start (first step only), then the ring's points.
      const int base = first ? 1 : 0, n = base + (ring ? pts : 0);
      const int lpc = lanes_per(n), sub = lane % lpc, c = lane / lpc;
      const int k = c - base;
      int mx = cmx, my = cmy;
      bool ok;
      if (k < 0) {
        ok = c < n;
      } else {
        const int kk = k & 7;
        mx = (int)(int16_t)(cmx + c_ring[kk][0] * step);
        my = (int)(int16_t)(cmy + c_ring[kk][1] * step);
        ok = c < n && mx >= qlx && mx <= qhx && my >= qly && my <= qhy &&
             !(has_prev && abs(mx - prevx) <= step && abs(my - prevy) <= step);
      }
      const int xi = B.x + (mx >> 2), yi = B.y + (my >> 2);
      const int8_t* q = c_h264_qpel[(my & 3) * 4 + (mx & 3)];
      const S* p1 = plane_at<S>(R, q[0], xi + q[1], yi + q[2]);
      const S* p2 = q[3] < 0 ? nullptr : plane_at<S>(R, q[3], xi + q[4], yi + q[5]);
      const uint32_t sv = group_satd<S>(sm.src, B.wr, B.tw, B.th, p1, p2, R.stride, lpc, sub, lane, ok);
      const uint32_t cost = ok ? sv + h264_rate(F, B, mx, my) : kInf;
      nsatd += __popc(__ballot_sync(kFull, ok && sub == 0));
      const Pick p = warp_min(cost);
      if (p.cost < bc) {
        bc = p.cost;
        bsatd = __shfl_sync(kFull, sv, p.lane);
        bmx = __shfl_sync(kFull, mx, p.lane);
        bmy = __shfl_sync(kFull, my, p.lane);
      }
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
  const bool ma = a.ref == ref, mb = b.ref == ref, mc = c.ref == ref;
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

// Returns a task it made ready to run next (frame << 24 | task), or -1.
template <class S>
__device__ int h264_task(const LaunchDesc& L, const FrameDesc& F, int f, int t, WarpSmem<S>& sm, int lane) {
  H264Blk B;
  uint32_t nsad = 0, nsatd = 0;
  int cont = -1;
  auto shape = [&](int x, int y, int w, int h) {  // search_bounds (h264_hpel.rs:476-488)
    B.x = x;
    B.y = y;
    B.w = w;
    B.h = h;
    B.lx = 4 - F.pad - x;
    B.hx = F.width + F.pad - (w + 4) - x;
    B.ly = max(4 - F.pad - y, -F.vr);
    B.hy = min(F.height + F.pad - (h + 4) - y, F.vr);
    B.wr = w * (int)sizeof(S) / 4;
    B.ipc = B.wr * h;
    B.tw = w >> 2;
    B.th = h >> 2;
    B.tpc = B.tw * B.th;
  };
  if (F.mode == RME_PRED_GIVEN) {
    const rme_job* j = &F.jobs[t];
    if (!given_job_ok(F, j, 8)) {  // p_mb's cands: at most 8
      if (lane == 0) atomicOr(L.status, kStatusBadTask);
      return -1;
    }
    shape(j->x, j->y, j->w, j->h);
    B.px = j->mvp[0].x;
    B.py = j->mvp[0].y;
    const int nc = j->nseeds;
    const int cx = lane >= 1 && lane - 1 < nc ? j->seeds[lane - 1].x : 0;
    const int cy = lane >= 1 && lane - 1 < nc ? j->seeds[lane - 1].y : 0;
    stage_src<S>(sm.src, plane_at<S>(F.src, 0, B.x, B.y), F.src.stride, B.w, B.h, lane);
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
    shape(mx * 16, my * 16, 16, 16);
    // Lanes 0..3 load the A, B, C, D neighbours' results together.
    int nqx = mx, nqy = my;
    if (lane == 0) nqx = mx - 1;
    if (lane == 1) nqy = my - 1;
    if (lane == 2) {
      nqx = mx + 1;
      nqy = my - 1;
    }
    if (lane == 3) {
      nqx = mx - 1;
      nqy = my - 1;
    }
    const bool nok = lane < 4 && nqx >= 0 && nqy >= 0 && nqx < mbw;
    uint32_t nmv = 0, nref = 0;
    if (nok) {
      nmv = ldcg_u32(&F.out[nqy * mbw + nqx].mv);
      nref = ldcg_u32(reinterpret_cast<const uint32_t*>(&F.out[nqy * mbw + nqx].ref));
    }
    const uint32_t navail = __ballot_sync(kFull, nok);
    auto nb = [&](int k) {
      Nb m{false, -1, 0, 0};
      const uint32_t v = __shfl_sync(kFull, nmv, k);
      const int rf = (int)__shfl_sync(kFull, nref, k);
      if (!((navail >> k) & 1u)) return m;
      m.avail = true;
      m.ref = rf;
      m.x = mvx_of(v);
      m.y = mvy_of(v);
      return m;
    };
    const Nb A = nb(0), Bn = nb(1), C = nb(2), D = nb(3);
    const Nb Cc = C.avail ? C : D;
    // p_skip_mv (h264/mb.rs:1235-1246)
    int skx = 0, sky = 0;
    if (A.avail && Bn.avail && !(A.ref == 0 && A.x == 0 && A.y == 0) && !(Bn.ref == 0 && Bn.x == 0 && Bn.y == 0))
      median_mvp(A, Bn, Cc, 0, skx, sky);
    // cands = [skip_mv, 0, distinct A, B, C vectors] (h264_pic.rs:713-751);
    // lane k + 1 holds candidate k.
    int ncx[8], ncy[8], nc = 0;
    ncx[nc] = skx;
    ncy[nc++] = sky;
    ncx[nc] = 0;
    ncy[nc++] = 0;
    {
      const Nb q[3] = {A, Bn, C};
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
    stage_src<S>(sm.src, plane_at<S>(F.src, 0, B.x, B.y), F.src.stride, 16, 16, lane);
    int mv16x = 0, mv16y = 0, r16 = 0, mi16x = 0, mi16y = 0;
    uint32_t c16 = kInf, s16 = 0, ci16 = 0, int16 = kInf;
    for (int r = 0; r < F.nref; ++r) {
      int prx, pry;
      median_mvp(A, Bn, Cc, r, prx, pry);
      if (r > 0 && nc < 8) {
        ncx[nc] = prx;
        ncy[nc] = pry;
      }
      const int k = r > 0 ? min(nc + 1, 8) : nc;
      B.px = prx;
      B.py = pry;
      int cx = 0, cy = 0;
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (lane == i + 1) {
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
    // The macroblocks whose A, B, C or D this one is, one per lane (the
    // warp barrier orders lane 0's result before the releasing atomics).
    const int mbh = F.height / 16;
    __syncwarp();
    bool rel = false;
    int dtask = 0;
    if (lane == 0) {
      rel = mx + 1 < mbw;
      dtask = t + 1;
    } else if (lane == 1) {
      rel = my + 1 < mbh && mx > 0;
      dtask = t + mbw - 1;
    } else if (lane == 2) {
      rel = my + 1 < mbh;
      dtask = t + mbw;
    } else if (lane == 3) {
      rel = my + 1 < mbh && mx + 1 < mbw;
      dtask = t + mbw + 1;
    }
    cont = release_lanes(L, F, f, rel, dtask, cont, lane);
  }
  count_task(sm, lane, nsad, nsatd, B.w * B.h);
  return cont;
}

}  // namespace
}  // namespace rme
