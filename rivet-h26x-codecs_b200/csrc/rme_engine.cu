// The resident engine: one search kernel that stays on the GPU while a
// serving loop feeds it, so frames that arrive while others are being
// searched join the running search instead of waiting for the next launch.
//
// A frame goes in through the upload stream, behind its source picture's
// upload: its descriptor into a slot of the device frame table, its
// finished count cleared, then a publish kernel pushes its work into the
// two rings (the warps' ring and the CTAs' ring). HEVC frames without AMP
// units go in the row form: every row of blocks of every level and
// reference is pushed at once, in an order where each row comes after the
// rows it reads, and the warp or CTA that takes a row searches its blocks
// left to right, waiting only for the published vectors of the row above
// and of the parent rows (rme_search_impl.cuh). Other frames go in the
// dataflow form: their dependency counts from the shape's template, their
// root tasks pushed, and each finished task pushing the tasks it makes
// ready. A warp takes a ring slot by ticket (the head's next index) and
// waits for it to be filled; the warp or CTA that completes a frame raises
// the frame's flag in mapped host memory; the host copies the results out
// and frees the slot.
//
// Pictures are refilled while the kernel runs (RME_PICTURES_CHANGE_IN_FLIGHT:
// reads of pictures use ordinary cached loads, never the read-only path),
// and a warp copies a frame's descriptor into its shared memory when it
// takes work of a frame it does not hold already.
//
// Waits are bounded: a slot or a published vector not yet written is waited
// for at most kSpinLimit polls (then the status word's timeout bit); waiting
// warps leave when the host sets the stop word (it does so only with no
// frame in flight), and the host launches the kernel again when work comes.
#define RME_PICTURES_CHANGE_IN_FLIGHT 1
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "rme_search_impl.cuh"

namespace rme {
namespace {

__device__ __forceinline__ uint32_t atom_add_release(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.release.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// A frame's completion, settled one task late (the count's atomic returns
// while the warp runs its next task, or while it waits for one): when this
// warp's increment was the frame's last, every result of the frame is
// visible to it; it makes them visible system-wide and raises the flag.
struct Settle {
  int f = -1;
  uint32_t old = 0, n = 0, gen = 0;
};
__device__ __forceinline__ void settle(const EngineCtl& E, Settle& st) {
  if (st.f >= 0 && st.old + 1u == st.n) {
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    __threadfence_system();
    E.hflags[st.f] = st.gen;
  }
  st.f = -1;
}

// Lane 0: the entry of the next slot of a ring (`big`: the CTAs' ring). The
// warp takes a ticket (the head's next index) and waits for that slot to be
// pushed, backing off to a microsecond between polls: a ticket per pop, so
// thousands of idle warps never contend on the head. Returns kPopDone when
// the host asks the kernel to leave (it does so only with nothing in flight,
// and resets the heads before launching it again), or 0xffffffff when the
// wait runs out (kSpinLimit polls: the status word's timeout bit).
__device__ __forceinline__ uint32_t engine_pop(const LaunchDesc& L, const EngineCtl& E, Settle& st, bool big,
                                               uint32_t& gen) {
  const unsigned long long idx = atomicAdd(big ? L.head_big : L.head, 1ull);
  const uint32_t lap = ring_lap(L.ring_shift, idx);
  const unsigned long long* slot = (big ? L.ready_big : L.ready) + (idx & ((1ull << L.ring_shift) - 1ull));
  uint32_t ns = 32;
  for (uint32_t it = 0;; ++it) {
    const unsigned long long v = ld_acquire64(slot);
    if ((uint32_t)(v >> 48) == lap) {
      gen = (uint32_t)(v >> 32) & 0xffffu;
      return (uint32_t)v;
    }
    settle(E, st);
    // The stop word is device memory: thousands of waiting warps polling a
    // host word would fill the bus the uploads and result copies use.
    if ((it & 7u) == 7u && ld_relaxed_gpu(E.stop) != 0u) return kPopDone;
    if (it >= kSpinLimit) {
      atomicOr(L.status, kStatusWaitTimeout);
      return 0xffffffffu;
    }
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
  }
}

// After the kernel has left: the next pop of each ring is the next push
// (tickets taken by warps that left unserved are dropped), and the stop
// word is cleared.
__global__ void reset_heads_kernel(LaunchDesc L, uint32_t* stop) {
  *L.head = *L.tail;
  *L.head_big = *L.tail_big;
  *stop = 0u;
}

// Registers: at most 112 a thread, so that the grid's two blocks per SM
// (57,344 registers) leave 8,192 on every SM to the kernels that run beside
// the resident one (plane builds in blocks of 128 threads, frame
// preparation and publication, each within that share). With 128, the
// engine would take every register of every SM, those kernels could not
// start until it left, and it leaves only once no frame is in flight: the
// frames queued behind them would never arrive.
constexpr int kEngineMaxRegs = 112;

// A CTA serving the ring of 32x32 and 64x64 HEVC blocks: all its threads
// run each task together (hevc_group_task).
template <class S>
__device__ void engine_group_task(const LaunchDesc& L, const FrameDesc& F, int f, int t, GroupSmem<S>& gs, int tid,
                                  int& cont) {
  const int blk = t / F.nref;
  int l = 0;
  while (l + 1 < F.nlevels && blk >= F.base[l + 1]) ++l;
  if (F.size[l] == 64) cont = hevc_group_task<S, 64>(L, F, f, t, gs, tid);
  else if (F.size[l] == 32) cont = hevc_group_task<S, 32>(L, F, f, t, gs, tid);
  else if (tid == 0) atomicOr(L.status, kStatusBadTask);
}

__device__ void engine_group_loop(const LaunchDesc& L, const EngineCtl& E, unsigned char* smem_raw, FrameDesc& F) {
  GroupSmem<uint16_t>& g16 = *reinterpret_cast<GroupSmem<uint16_t>*>(smem_raw);
  GroupSmem<uint8_t>& g8 = *reinterpret_cast<GroupSmem<uint8_t>*>(smem_raw);
  const int tid = threadIdx.x;
  if (tid < 6) g16.cnt[tid] = 0;
  __syncthreads();
  Settle st;
  int cont = -1;
  int cached = -1;  // the frame slot whose descriptor F holds (generation in cached_gen)
  uint32_t cached_gen = 0;
  for (;;) {
    uint32_t e;
    if (cont >= 0) {
      e = (uint32_t)cont;
    } else {
      if (tid == 0) {
        uint32_t gen = 0;
        g16.bc[7] = engine_pop(L, E, st, true, gen);
        g16.bc[5] = gen;
      }
      __syncthreads();
      e = g16.bc[7];
      const uint32_t gen = g16.bc[5];
      // The descriptor is copied through L2 unless this CTA holds it already.
      if (e != kPopDone && e != 0xffffffffu && ((int)(e >> 24) != cached || gen != cached_gen)) {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&L.frames[e >> 24]);
        uint32_t* to = reinterpret_cast<uint32_t*>(&F);
        for (int i = tid; i < (int)(sizeof(FrameDesc) / 4); i += kGroupThreads) to[i] = __ldcg(from + i);
        cached = (int)(e >> 24);
        cached_gen = gen;
      }
      __syncthreads();
      if (e == kPopDone) break;
    }
    cont = -1;
    if (e == 0xffffffffu) continue;
    const int f = (int)(e >> 24), t = (int)(e & 0xffffffu);
    if (F.mvf != nullptr) {  // a row of the frame's 32x32 or 64x64 blocks
      if (F.bd == 8) hevc_group_row<uint8_t>(L, F, f, (uint32_t)t, g8, tid);
      else hevc_group_row<uint16_t>(L, F, f, (uint32_t)t, g16, tid);
    } else if (t >= F.ntasks || !group_task_of(L, F, t)) {
      if (tid == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    } else if (F.bd == 8) {
      engine_group_task<uint8_t>(L, F, f, t, g8, tid, cont);
    } else {
      engine_group_task<uint16_t>(L, F, f, t, g16, tid, cont);
    }
    if (tid == 0) {
      settle(E, st);
      st.old = atom_add_release(&E.fdone[f], 1u);  // thread 0 wrote the results itself
      st.f = f;
      st.n = (uint32_t)(F.mvf != nullptr ? F.nrows : F.ntasks);
      st.gen = F.gen;
    }
  }
  if (tid == 0) settle(E, st);
  __syncthreads();
  if (tid < 5) atomicAdd(&L.counters[tid], g16.cnt[tid]);
}

__global__ void __maxnreg__(kEngineMaxRegs) engine_kernel(LaunchDesc L, EngineCtl E) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FrameDesc fdesc[kWarpsPerBlock];
  if ((int)blockIdx.x < L.group_ctas) {
    engine_group_loop(L, E, smem_raw, fdesc[0]);
    return;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem<uint16_t>& sm16 = reinterpret_cast<WarpSmem<uint16_t>*>(smem_raw)[warp];
  WarpSmem<uint8_t>& sm8 = reinterpret_cast<WarpSmem<uint8_t>&>(sm16);
  FrameDesc& F = fdesc[warp];
  if (lane < 6) sm16.cnt[lane] = 0;
  __syncwarp();
  Settle st;
  int cont = -1;
  int cached = -1;  // the frame slot whose descriptor F holds (generation in cached_gen)
  uint32_t cached_gen = 0;
  for (;;) {
    uint32_t e;
    if (cont >= 0) {
      e = (uint32_t)cont;  // a task of the same frame: its descriptor is here already
    } else {
      e = 0;
      uint32_t gen = 0;
      if (lane == 0) e = engine_pop(L, E, st, false, gen);
      e = __shfl_sync(kFull, e, 0);
      gen = __shfl_sync(kFull, gen, 0);
      if (e == kPopDone) break;
      // The descriptor is copied through L2 unless this warp holds it already.
      if (e != 0xffffffffu && ((int)(e >> 24) != cached || gen != cached_gen)) {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&L.frames[e >> 24]);
        uint32_t* to = reinterpret_cast<uint32_t*>(&F);
        for (int i = lane; i < (int)(sizeof(FrameDesc) / 4); i += 32) to[i] = __ldcg(from + i);
        cached = (int)(e >> 24);
        cached_gen = gen;
      }
    }
    __syncwarp();
    cont = -1;
    if (e == 0xffffffffu) continue;
    const int f = (int)(e >> 24), t = (int)(e & 0xffffffu);
    if (F.mvf != nullptr) {  // a row of the frame's 16x16 or 8x8 blocks
      if (F.bd == 8) hevc_row<uint8_t, true>(L, F, f, (uint32_t)t, sm8, lane);
      else hevc_row<uint16_t, true>(L, F, f, (uint32_t)t, sm16, lane);
    } else if (t >= F.ntasks || F.mode != RME_PRED_STANDALONE) {
      if (lane == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    } else if (F.codec == RME_CODEC_HEVC) {
      cont = F.bd == 8 ? hevc_task<uint8_t, true>(L, F, f, t, sm8, lane) : hevc_task<uint16_t, true>(L, F, f, t, sm16, lane);
    } else {
      cont = F.bd == 8 ? h264_task<uint8_t>(L, F, f, t, sm8, lane) : h264_task<uint16_t>(L, F, f, t, sm16, lane);
    }
    if (lane == 0) {
      settle(E, st);
      // Release: lane 0 wrote the results itself.
      st.old = atom_add_release(&E.fdone[f], 1u);
      st.f = f;
      st.n = (uint32_t)(F.mvf != nullptr ? F.nrows : F.ntasks);
      st.gen = F.gen;
    }
  }
  if (lane == 0) settle(E, st);
  __syncwarp();
  if (lane < 5) atomicAdd(&L.counters[lane], sm16.cnt[lane]);
}

// A frame's root tasks (those that read no other task's result) into their
// rings, queued behind everything the frame needs (its descriptor among it).
__global__ void publish_kernel(LaunchDesc L, int f, const uint32_t* roots, int n) {
  const FrameDesc& F = L.frames[f];
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    push_ready(L, f, (int)roots[i], group_task_of(L, F, (int)roots[i]), F.gen);
}

// A row-form frame's rows into the two rings, each list in its order: one
// reservation of consecutive slots per ring, so that every row is popped
// after the rows it reads.
__global__ void publish_rows_kernel(LaunchDesc L, int f, const uint32_t* rows, int n, const uint32_t* rows_big,
                                    int nbig) {
  __shared__ unsigned long long base[2];
  const uint32_t gen = L.frames[f].gen;
  if (threadIdx.x == 0) {
    base[0] = atomicAdd(L.tail, (unsigned long long)n);
    base[1] = atomicAdd(L.tail_big, (unsigned long long)nbig);
  }
  __syncthreads();
  const unsigned long long mask = (1ull << L.ring_shift) - 1ull;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const unsigned long long idx = base[0] + i;
    st_release64(L.ready + (idx & mask), ring_entry(L.ring_shift, idx, gen, f, (int)rows[i]));
  }
  for (int i = threadIdx.x; i < nbig; i += blockDim.x) {
    const unsigned long long idx = base[1] + i;
    st_release64(L.ready_big + (idx & mask), ring_entry(L.ring_shift, idx, gen, f, (int)rows_big[i]));
  }
}

// A frame's dependency counts from its shape's template into its slot, its
// finished count cleared, and (a row-form frame's fresh buffer) its
// published words zeroed: a kernel (beside the resident one) rather than
// device copies and memsets, which the driver may run as kernels of its own
// that would wait for the resident kernel to leave.
__global__ void prepare_kernel(int32_t* pending, const int32_t* tmpl, int n, uint32_t* fdone,
                               unsigned long long* zero, int64_t nzero) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = i; k < n; k += gridDim.x * blockDim.x) pending[k] = tmpl[k];
  for (int64_t k = i; k < nzero; k += gridDim.x * blockDim.x) zero[k] = 0ull;
  if (i == 0) *fdone = 0u;
}

size_t engine_smem() { return sizeof(WarpSmem<uint16_t>) * kWarpsPerBlock; }

}  // namespace

int engine_blocks_per_sm() {
  int n = 0;
  cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)engine_smem());
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, engine_kernel, kWarpsPerBlock * 32, engine_smem());
  return e == cudaSuccess && n > 0 ? n : 1;
}

cudaError_t launch_engine(const LaunchDesc& L, const EngineCtl& E, int grid, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)engine_smem());
  if (e != cudaSuccess) return e;
  prefer_max_shared(engine_kernel);
  engine_kernel<<<grid, kWarpsPerBlock * 32, engine_smem(), s>>>(L, E);
  return cudaGetLastError();
}

static cudaError_t launch_prepare(int32_t* pending, const int32_t* tmpl, int n, uint32_t* fdone,
                                  unsigned long long* zero, int64_t nzero, cudaStream_t s) {
  prefer_max_shared(prepare_kernel);
  const int64_t most = std::max<int64_t>(n, nzero);
  prepare_kernel<<<(int)std::min<int64_t>(64, (most + 255) / 256 + 1), 256, 0, s>>>(pending, tmpl, n, fdone, zero,
                                                                                    nzero);
  return cudaGetLastError();
}

static cudaError_t launch_publish_rows(const LaunchDesc& L, int frame, const uint32_t* rows, int n,
                                       const uint32_t* rows_big, int nbig, cudaStream_t s) {
  prefer_max_shared(publish_rows_kernel);
  publish_rows_kernel<<<1, 256, 0, s>>>(L, frame, rows, n, rows_big, nbig);
  return cudaGetLastError();
}

cudaError_t launch_publish(const LaunchDesc& L, int frame, const uint32_t* roots, int nroots, cudaStream_t s) {
  prefer_max_shared(publish_kernel);
  publish_kernel<<<1, 256, 0, s>>>(L, frame, roots, nroots);
  return cudaGetLastError();
}

// ---- host side ------------------------------------------------------------------

namespace {
constexpr int kRingShift = 22;  // 4 Mi slots (32 MiB): the tasks in flight at once
constexpr int kHdrHead = 0, kHdrTail = 1, kHdrStatus = 2, kHdrCounters = 3, kHdrEpoch = 8, kHdrHeadBig = 9,
              kHdrTailBig = 10, kHdrStop = 11, kHdrWords = 16;
}  // namespace

struct EngineSlot {
  bool busy = false;
  uint32_t gen = 0;
  int ntasks = 0;
  rme_result* d_out = nullptr;
  size_t out_cap = 0;
  int32_t* d_pending = nullptr;
  size_t pend_cap = 0;
  unsigned long long* d_mvf = nullptr;  // the row form's published words
  size_t mvf_cap = 0;
};

struct Engine {
  void* ctx = nullptr;
  int device = 0, grid = 0;
  unsigned long long* d_hdr = nullptr;
  unsigned long long* d_ring = nullptr;  // the warps' ring, then the CTAs' ring
  FrameDesc* d_frames = nullptr;
  FrameDesc* h_frames = nullptr;  // pinned: each slot's descriptor, copied at submit
  uint32_t* d_fdone = nullptr;
  uint32_t* h_flags = nullptr;    // mapped pinned: per slot, the generation finished
  uint32_t* dh_flags = nullptr;   // their device address
  uint32_t* h_one = nullptr;      // pinned: the stop word's value, copied into device memory to stop the kernel
  cudaStream_t kstream = nullptr, ctl = nullptr;
  cudaEvent_t ended = nullptr;
  bool launched = false;
  int64_t launches = 0;  // kernel launches (it leaves when idle)
  EngineSlot slots[kEngineFrames];
  std::vector<int> free_slots;
  int64_t inflight_tasks = 0;
  std::vector<void*> outgrown;  // device buffers replaced while the kernel could run (freed at the end)
  LaunchDesc L{};
  EngineCtl E{};
};

void engine_destroy(Engine* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->launched && !engine_idle(g) && g->ctl && g->h_one) {
    // The warps leave (waiting ones within microseconds).
    cudaMemcpyAsync(g->d_hdr + kHdrStop, g->h_one, sizeof(uint32_t), cudaMemcpyHostToDevice, g->ctl);
    cudaEventSynchronize(g->ended);
  }
  cudaDeviceSynchronize();
  for (auto& s : g->slots) {
    if (s.d_out) cudaFree(s.d_out);
    if (s.d_pending) cudaFree(s.d_pending);
    if (s.d_mvf) cudaFree(s.d_mvf);
  }
  for (void* p : g->outgrown) cudaFree(p);
  if (g->d_hdr) cudaFree(g->d_hdr);
  if (g->d_ring) cudaFree(g->d_ring);
  if (g->d_frames) cudaFree(g->d_frames);
  if (g->h_frames) cudaFreeHost(g->h_frames);
  if (g->d_fdone) cudaFree(g->d_fdone);
  if (g->h_flags) cudaFreeHost(g->h_flags);
  if (g->h_one) cudaFreeHost(g->h_one);
  if (g->ctl) cudaStreamDestroy(g->ctl);
  if (g->ended) cudaEventDestroy(g->ended);
  if (g->kstream) cudaStreamDestroy(g->kstream);
  delete g;
}

int engine_create(void* ctx, int device, Engine** out) {
  auto* g = new Engine();
  g->ctx = ctx;
  g->device = device;
  cudaError_t e = cudaSetDevice(device);
  int nsm = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_hdr, kHdrWords * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(g->d_hdr, 0, kHdrWords * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&g->d_ring, 2 * (sizeof(unsigned long long) << kRingShift));
  // Slot words start at zero: lap tags start at 1.
  if (e == cudaSuccess) e = cudaMemset(g->d_ring, 0, 2 * (sizeof(unsigned long long) << kRingShift));
  if (e == cudaSuccess) e = cudaMalloc(&g->d_frames, sizeof(FrameDesc) * kEngineFrames);
  if (e == cudaSuccess) e = cudaMemset(g->d_frames, 0, sizeof(FrameDesc) * kEngineFrames);
  if (e == cudaSuccess) e = cudaMallocHost(&g->h_frames, sizeof(FrameDesc) * kEngineFrames);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_fdone, sizeof(uint32_t) * kEngineFrames);
  if (e == cudaSuccess) e = cudaHostAlloc(&g->h_flags, sizeof(uint32_t) * kEngineFrames, cudaHostAllocMapped);
  if (e == cudaSuccess) {
    std::memset(g->h_flags, 0, sizeof(uint32_t) * kEngineFrames);
    e = cudaHostGetDevicePointer((void**)&g->dh_flags, g->h_flags, 0);
  }
  if (e == cudaSuccess) e = cudaMallocHost(&g->h_one, 64);
  if (e == cudaSuccess) *g->h_one = 1u;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->ctl, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->kstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ended, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    engine_destroy(g);
    return RME_ECUDA;
  }
  // At most two of the kernel's blocks per SM: room is left on every SM for
  // the uploads' plane builds, which run beside it.
  g->grid = nsm * std::min(2, engine_blocks_per_sm());
  // Half of them run the 32x32 and 64x64 HEVC blocks (a CTA per block, or
  // per row of blocks in the row form), the other half's warps the smaller
  // blocks: a 1080p frame of two references has 98 rows of large blocks and
  // 404 of small ones (a frame measured 5.6 ms this way, 6.2 ms with two
  // thirds of the CTAs on large blocks).
  const int groups = std::max(1, g->grid / 2);
  for (int k = kEngineFrames - 1; k >= 0; --k) g->free_slots.push_back(k);
  LaunchDesc& L = g->L;
  L.frames = g->d_frames;
  L.ready = g->d_ring;
  L.total = 1ll << kRingShift;
  L.head = g->d_hdr + kHdrHead;
  L.tail = g->d_hdr + kHdrTail;
  L.status = reinterpret_cast<uint32_t*>(g->d_hdr + kHdrStatus);
  L.counters = g->d_hdr + kHdrCounters;
  L.epoch = reinterpret_cast<const uint32_t*>(g->d_hdr + kHdrEpoch);
  L.done = nullptr;
  L.ready_big = g->d_ring + (1ull << kRingShift);
  L.head_big = g->d_hdr + kHdrHeadBig;
  L.tail_big = g->d_hdr + kHdrTailBig;
  L.group_ctas = groups;
  L.patch8 = 1;
  L.ring_shift = kRingShift;
  EngineCtl& E = g->E;
  E.fdone = g->d_fdone;
  E.hflags = g->dh_flags;
  E.stop = reinterpret_cast<const uint32_t*>(g->d_hdr + kHdrStop);
  E.idle_polls = 0u;  // unused: the host stops the kernel when it has been idle
  *out = g;
  return 0;
}

bool engine_idle(Engine* g) {
  if (!g->launched) return true;
  const cudaError_t e = cudaEventQuery(g->ended);
  cudaGetLastError();
  return e != cudaErrorNotReady;
}

// The kernel runs, or is launched again (it leaves once idle).
static int engine_run(Engine* g) {
  if (!engine_idle(g)) return 0;
  if (launch_engine(g->L, g->E, g->grid, g->kstream) != cudaSuccess) return RME_ECUDA;
  if (cudaEventRecord(g->ended, g->kstream) != cudaSuccess) return RME_ECUDA;
  g->launched = true;
  ++g->launches;
  return 0;
}

int engine_submit(Engine* g, const rme_frame* f, const rme_params* p, cudaStream_t upload, int* slot_out) {
  FrameDesc fd;
  int ntasks = 0, nroots = 0;
  const int32_t* tmpl = nullptr;
  const uint32_t* roots = nullptr;
  int rc = ctx_standalone_frame(g->ctx, f, p, &fd, &ntasks, &tmpl, &roots, &nroots);
  if (rc) return rc;
  if (g->free_slots.empty() || g->inflight_tasks + ntasks > (1ll << kRingShift)) return RME_EBUSY;
  // HEVC frames without AMP run in the row form.
  const uint32_t *rows = nullptr, *rows_big = nullptr;
  int nrows = 0, nrows_big = 0;
  const bool row_form = ctx_frame_rows(g->ctx, f, p, &rows, &nrows, &rows_big, &nrows_big);
  const int k = g->free_slots.back();
  EngineSlot& s = g->slots[k];
  if (s.out_cap < (size_t)ntasks) {
    if (s.d_out) g->outgrown.push_back(s.d_out);
    s.d_out = nullptr;
    s.out_cap = 0;
    if (cudaMalloc(&s.d_out, sizeof(rme_result) * ntasks) != cudaSuccess) return RME_ENOMEM;
    s.out_cap = ntasks;
  }
  if (!row_form && s.pend_cap < (size_t)ntasks) {
    if (s.d_pending) g->outgrown.push_back(s.d_pending);
    s.d_pending = nullptr;
    s.pend_cap = 0;
    if (cudaMalloc(&s.d_pending, sizeof(int32_t) * ntasks) != cudaSuccess) return RME_ENOMEM;
    s.pend_cap = ntasks;
  }
  // A fresh buffer of published words is zeroed (generations start at 1).
  int64_t nzero = 0;
  if (row_form && s.mvf_cap < (size_t)ntasks) {
    if (s.d_mvf) g->outgrown.push_back(s.d_mvf);
    s.d_mvf = nullptr;
    s.mvf_cap = 0;
    if (cudaMalloc(&s.d_mvf, sizeof(unsigned long long) * ntasks) != cudaSuccess) return RME_ENOMEM;
    s.mvf_cap = ntasks;
    nzero = ntasks;
  }
  if (++s.gen == 0) s.gen = 1;
  fd.out = s.d_out;
  fd.pending = row_form ? nullptr : s.d_pending;
  fd.gen = s.gen;
  if (row_form) {
    fd.mvf = s.d_mvf;
    fd.tag = s.gen;
    fd.nrows = nrows + nrows_big;
  }
  g->h_frames[k] = fd;
  if (launch_prepare(row_form ? nullptr : s.d_pending, tmpl, row_form ? 0 : ntasks, g->d_fdone + k, s.d_mvf, nzero,
                     upload) != cudaSuccess ||
      cudaMemcpyAsync(g->d_frames + k, g->h_frames + k, sizeof(FrameDesc), cudaMemcpyHostToDevice, upload) !=
          cudaSuccess ||
      (row_form ? launch_publish_rows(g->L, k, rows, nrows, rows_big, nrows_big, upload)
                : launch_publish(g->L, k, roots, nroots, upload)) != cudaSuccess)
    return RME_ECUDA;
  g->free_slots.pop_back();
  s.busy = true;
  s.ntasks = ntasks;
  g->inflight_tasks += ntasks;
  *slot_out = k;
  return engine_run(g);
}

// Stop the kernel (nothing in flight): ask its warps to leave, wait, reset
// the heads. The next submit launches it again.
int engine_stop(Engine* g) {
  if (!g->launched || engine_idle(g)) return 0;
  if (g->inflight_tasks > 0) return RME_EBUSY;
  cudaError_t e =
      cudaMemcpyAsync(g->d_hdr + kHdrStop, g->h_one, sizeof(uint32_t), cudaMemcpyHostToDevice, g->ctl);
  if (e == cudaSuccess) e = cudaEventSynchronize(g->ended);
  if (e == cudaSuccess) {
    prefer_max_shared(reset_heads_kernel);
    reset_heads_kernel<<<1, 1, 0, g->kstream>>>(g->L, reinterpret_cast<uint32_t*>(g->d_hdr + kHdrStop));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->kstream);
  return e == cudaSuccess ? 0 : RME_ECUDA;
}

bool engine_done(Engine* g, int slot) {
  return ((volatile uint32_t*)g->h_flags)[slot] == g->slots[slot].gen;
}

// The kernel left (idle) while frames were in flight: launch it again.
int engine_keep_running(Engine* g) { return g->inflight_tasks > 0 ? engine_run(g) : 0; }

const rme_result* engine_results(Engine* g, int slot) { return g->slots[slot].d_out; }
int engine_slot_tasks(Engine* g, int slot) { return g->slots[slot].ntasks; }
const uint32_t* engine_status_word(Engine* g) { return reinterpret_cast<const uint32_t*>(g->d_hdr + kHdrStatus); }

void engine_release(Engine* g, int slot) {
  EngineSlot& s = g->slots[slot];
  if (!s.busy) return;
  s.busy = false;
  g->inflight_tasks -= s.ntasks;
  g->free_slots.push_back(slot);
}

}  // namespace rme
