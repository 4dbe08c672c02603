// The motion search on the device: one persistent launch per kind of task
// (sample width, codec), one warp per (block, reference) task, tasks pulled
// from a device work queue.
//
// What a task computes is the reference's search, step for step:
//   HEVC   search_full   (encode/h265_me.rs:3749-3858): seeds floored to
//          whole samples (arithmetic >> 2), clamp_pos to +-(pad - MARGIN), deduplicated
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
//
// The reference scores one candidate at a time and takes it when strictly
// cheaper than the best so far. Every candidate of a step is known before
// the step (each ring is around a centre fixed for the step), so here a
// warp scores them together: a group of lanes per candidate computes its
// distortion and its rate, and the step's outcome is the warp minimum —
// the lowest-indexed candidate among those of least cost, taken when below
// the best. That is exactly the sequential strict-< walk: it ends on the
// least cost, and on the first candidate reaching it.
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
// block one size up; H.264: the A, B, C and D macroblocks). Each task has a
// count of those; a finishing task decrements its readers' counts and
// pushes onto the launch's ready queue each one it brings to zero, so a
// warp only ever takes a task whose inputs are complete. The only wait is
// for the queue itself (a slot not yet pushed: nothing is ready anywhere);
// it is bounded (kSpinLimit polls with backoff), and a wait that runs out
// sets a status bit the host turns into RME_EDEVICE instead of hanging.
#include <algorithm>

#include "rme_search_impl.cuh"

namespace rme {
namespace {

// One kernel per (sample width, codec, occupancy variant): a launch holds
// the tasks of one kind, so each kernel carries only its codec's search (a
// smaller body stays resident in the instruction caches). MINB is the
// number of resident blocks the register allocation is bounded for: 2
// leaves more registers per thread (a single frame's dependency chain runs
// faster), 4 keeps more warps resident (large batches hide more latency);
// the host's tuner picks per kind and launch size.
// A CTA of the latency form serving the queue of 32x32 and 64x64 blocks:
// all its threads run each task together (hevc_group_task).
template <class S>
__device__ void group_loop(const LaunchDesc& L, unsigned char* smem_raw) {
  GroupSmem<S>& gs = *reinterpret_cast<GroupSmem<S>*>(smem_raw);
  const int tid = threadIdx.x;
  if (tid < 6) gs.cnt[tid] = 0;
  const uint32_t epoch = __ldg(L.epoch);
  int cont = -1;
  __syncthreads();
  for (;;) {
    uint32_t e;
    if (cont >= 0) {
      e = (uint32_t)cont;
    } else {
      if (tid == 0) {
        const unsigned long long idx = atomicAdd(L.head_big, 1ull);
        gs.bc[7] = idx >= (unsigned long long)L.total ? kPopDone : pop_slot(L, idx, epoch, true);
      }
      __syncthreads();
      e = gs.bc[7];
      __syncthreads();
      if (e == kPopDone) break;
    }
    cont = -1;
    if (e == 0xffffffffu) continue;  // the wait ran out (status set)
    const int f = (int)(e >> 24), t = (int)(e & 0xffffffu);
    const FrameDesc& F = L.frames[f];
    if (t >= F.ntasks || (sizeof(S) == 1) != (F.bd == 8) || !group_task_of(L, F, t)) {
      if (tid == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    }
    const int blk = t / F.nref;
    int l = 0;
    while (l + 1 < F.nlevels && blk >= F.base[l + 1]) ++l;
    if (F.size[l] == 64) cont = hevc_group_task<S, 64>(L, F, f, t, gs, tid);
    else if (F.size[l] == 32) cont = hevc_group_task<S, 32>(L, F, f, t, gs, tid);
    else if (tid == 0) atomicOr(L.status, kStatusBadTask);
    if (tid == 0 && L.done != nullptr) red_add64(L.done, 1ull);
  }
  __syncthreads();
  if (tid < 5) atomicAdd(&L.counters[tid], gs.cnt[tid]);
}

// The row form: a CTA takes rows of 32x32 or 64x64 blocks (hevc_group_row)
// from the CTAs' queue, a warp rows of 16x16 or 8x8 blocks (hevc_row) from
// the warps' queue, until each queue is empty. The host pushed every row, in
// an order where each comes after the rows it reads, so a row's owner only
// waits for rows that are owned already.
template <class S>
__device__ void group_row_loop(const LaunchDesc& L, unsigned char* smem_raw) {
  GroupSmem<S>& gs = *reinterpret_cast<GroupSmem<S>*>(smem_raw);
  const int tid = threadIdx.x;
  if (tid < 6) gs.cnt[tid] = 0;
  const uint32_t epoch = __ldg(L.epoch);
  __syncthreads();
  for (;;) {
    if (tid == 0) {
      const unsigned long long idx = atomicAdd(L.head_big, 1ull);
      gs.bc[7] = idx >= (unsigned long long)L.total_big ? kPopDone : pop_slot(L, idx, epoch, true);
    }
    __syncthreads();
    const uint32_t e = gs.bc[7];
    __syncthreads();
    if (e == kPopDone) break;
    if (e == 0xffffffffu) continue;
    const int f = (int)(e >> 24);
    const FrameDesc& F = L.frames[f];
    if ((sizeof(S) == 1) != (F.bd == 8)) {
      if (tid == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    }
    hevc_group_row<S>(L, F, f, e & 0xffffffu, gs, tid);
  }
  __syncthreads();
  if (tid < 5) atomicAdd(&L.counters[tid], gs.cnt[tid]);
}

template <class S, bool SPEC>
__device__ void row_loop(const LaunchDesc& L, WarpSmem<S>& sm, int lane) {
  const uint32_t epoch = __ldg(L.epoch);
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(L.head, 1ull);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= (unsigned long long)L.total) break;
    uint32_t e = 0;
    if (lane == 0) e = pop_slot(L, idx, epoch);
    e = __shfl_sync(kFull, e, 0);
    if (e == 0xffffffffu) continue;
    const int f = (int)(e >> 24);
    const FrameDesc& F = L.frames[f];
    if ((sizeof(S) == 1) != (F.bd == 8)) {
      if (lane == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    }
    hevc_row<S, SPEC>(L, F, f, e & 0xffffffu, sm, lane);
  }
}

template <class S, int CODEC, int MINB, bool SPEC>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, MINB) search_kernel(LaunchDesc L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if constexpr (SPEC && CODEC == RME_CODEC_HEVC) {
    if (L.rows) {
      if ((int)blockIdx.x < L.group_ctas) {
        group_row_loop<S>(L, smem_raw);
      } else {
        const int lane = threadIdx.x & 31;
        WarpSmem<S>& sm = reinterpret_cast<WarpSmem<S>*>(smem_raw)[threadIdx.x >> 5];
        if (lane < 5) sm.cnt[lane] = 0;
        __syncwarp();
        row_loop<S, SPEC>(L, sm, lane);
        __syncwarp();
        if (lane < 5) atomicAdd(&L.counters[lane], sm.cnt[lane]);
      }
      return;
    }
    if ((int)blockIdx.x < L.group_ctas) {
      group_loop<S>(L, smem_raw);
      return;
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem<S>& sm = reinterpret_cast<WarpSmem<S>*>(smem_raw)[warp];
  if (lane < 5) sm.cnt[lane] = 0;
  __syncwarp();
  const uint32_t epoch = __ldg(L.epoch);
  int cont = -1;  // a task the last one made ready, run next by this warp
  for (;;) {
    uint32_t e;
    if (cont >= 0) {
      e = (uint32_t)cont;
    } else {
      unsigned long long idx = 0;
      if (lane == 0) idx = atomicAdd(L.head, 1ull);
      idx = __shfl_sync(kFull, idx, 0);
      if (idx >= (unsigned long long)L.total) break;
      e = 0;
      if (lane == 0) e = pop_slot(L, idx, epoch);
      e = __shfl_sync(kFull, e, 0);
      if (e == kPopDone) break;
    }
    __syncwarp();
    cont = -1;
    if (e == 0xffffffffu) continue;  // the wait ran out (status set)
    const int f = (int)(e >> 24), t = (int)(e & 0xffffffu);
    const FrameDesc& F = L.frames[f];
    // A task of another kind, or past its frame, is a host bug: flag it
    // and skip it rather than read out of bounds.
    if (t >= F.ntasks || (sizeof(S) == 1) != (F.bd == 8) || F.codec != CODEC) {
      if (lane == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    }
    if constexpr (CODEC == RME_CODEC_HEVC) cont = hevc_task<S, SPEC>(L, F, f, t, sm, lane);
    else cont = h264_task<S>(L, F, f, t, sm, lane);
    if (lane == 0 && L.done != nullptr) red_add64(L.done, 1ull);
  }
  __syncwarp();
  if (lane < 5) atomicAdd(&L.counters[lane], sm.cnt[lane]);
}

template <class S>
size_t smem_bytes() {
  return sizeof(WarpSmem<S>) * kWarpsPerBlock;
}

template <class S, int CODEC, int MINB, bool SPEC>
int blocks_per_sm() {
  int n = 0;
  cudaError_t e = cudaFuncSetAttribute(search_kernel<S, CODEC, MINB, SPEC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<S>());
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, search_kernel<S, CODEC, MINB, SPEC>, kWarpsPerBlock * 32,
                                                      smem_bytes<S>());
  return e == cudaSuccess && n > 0 ? n : 1;
}

// The shared-memory share of the SM's unified L1 that MINB blocks need
// (percent, rounded up): the rest stays L1 data cache, which the
// reference reads hit (a frame 3.9 -> 3.75 ms, an 8-frame launch 15.1 ->
// 14.0 ms against the largest shared share).
template <class S, int MINB>
int carveout_pct() {
  static int pct = -1;
  if (pct < 0) {
    int dev = 0, smem_sm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        smem_sm <= 0) {
      cudaGetLastError();
      return 100;
    }
    const long need = (long)MINB * ((long)smem_bytes<S>() + 1024);
    pct = (int)std::min<long>(100, (need * 100 + smem_sm - 1) / smem_sm);
  }
  return pct;
}

template <class S, int CODEC, int MINB, bool SPEC>
cudaError_t launch(const LaunchDesc& L, int grid, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(search_kernel<S, CODEC, MINB, SPEC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<S>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(search_kernel<S, CODEC, MINB, SPEC>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           carveout_pct<S, MINB>());
  if (e != cudaSuccess) return e;
  search_kernel<S, CODEC, MINB, SPEC><<<grid, kWarpsPerBlock * 32, smem_bytes<S>(), s>>>(L);
  return cudaGetLastError();
}

// The latency kernels (SPEC) exist for HEVC only; H.264 runs its one form.
template <class S, int CODEC, bool SPEC>
int bps_variant(int v) {
  return v == 0 ? blocks_per_sm<S, CODEC, 2, SPEC>() : v == 2 ? blocks_per_sm<S, CODEC, 4, SPEC>()
                                                              : blocks_per_sm<S, CODEC, 3, SPEC>();
}
template <class S, int CODEC, bool SPEC>
cudaError_t launch_variant(const LaunchDesc& L, int v, int grid, cudaStream_t s) {
  return v == 0 ? launch<S, CODEC, 2, SPEC>(L, grid, s) : v == 2 ? launch<S, CODEC, 4, SPEC>(L, grid, s)
                                                                 : launch<S, CODEC, 3, SPEC>(L, grid, s);
}

}  // namespace

int search_blocks_per_sm(int bytes_per_sample, int codec, int variant, bool spec) {
  if (codec == RME_CODEC_HEVC) {
    if (spec)
      return bytes_per_sample == 1 ? bps_variant<uint8_t, RME_CODEC_HEVC, true>(variant)
                                   : bps_variant<uint16_t, RME_CODEC_HEVC, true>(variant);
    return bytes_per_sample == 1 ? bps_variant<uint8_t, RME_CODEC_HEVC, false>(variant)
                                 : bps_variant<uint16_t, RME_CODEC_HEVC, false>(variant);
  }
  return bytes_per_sample == 1 ? bps_variant<uint8_t, RME_CODEC_H264, false>(variant)
                               : bps_variant<uint16_t, RME_CODEC_H264, false>(variant);
}

cudaError_t launch_search(const LaunchDesc& L, int bytes_per_sample, int codec, int variant, int grid, cudaStream_t s,
                          bool spec) {
  if (codec == RME_CODEC_HEVC) {
    if (spec)
      return bytes_per_sample == 1 ? launch_variant<uint8_t, RME_CODEC_HEVC, true>(L, variant, grid, s)
                                   : launch_variant<uint16_t, RME_CODEC_HEVC, true>(L, variant, grid, s);
    return bytes_per_sample == 1 ? launch_variant<uint8_t, RME_CODEC_HEVC, false>(L, variant, grid, s)
                                 : launch_variant<uint16_t, RME_CODEC_HEVC, false>(L, variant, grid, s);
  }
  return bytes_per_sample == 1 ? launch_variant<uint8_t, RME_CODEC_H264, false>(L, variant, grid, s)
                               : launch_variant<uint16_t, RME_CODEC_H264, false>(L, variant, grid, s);
}

}  // namespace rme
