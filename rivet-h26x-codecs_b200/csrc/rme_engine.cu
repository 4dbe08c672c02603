// The resident engine: one search kernel that stays on the GPU while a
// serving loop feeds it, so frames that arrive while others are being
// searched join the running search instead of waiting for the next launch.
//
// A frame goes in through the upload stream, behind its picture upload and
// plane builds: its descriptor into a slot of the device frame table, its
// dependency counts from the shape's template, its finished-task count
// cleared, then publish_kernel pushes its root tasks into the ring. Warps of
// the engine kernel claim pushed slots (compare-and-swap of the head below
// the tail: a warp never holds a slot that is not yet pushed, so warps may
// leave at any time without stranding work), run the same task functions as
// the batched kernels (rme_search_impl.cuh; STANDALONE rule, latency form),
// and push the tasks their results make ready. The warp whose task completes
// a frame raises the frame's flag in mapped host memory; the host copies the
// results out and frees the slot.
//
// Pictures are refilled while the kernel runs, so in this file every read of
// a picture goes through L2 (RME_PICTURES_CHANGE_IN_FLIGHT), and a warp
// copies a frame's descriptor into its shared memory through L2 when it
// takes a task of a frame from the ring.
//
// Waits are bounded: a claimed slot not yet written is waited for at most
// kSpinLimit polls (then the status word's timeout bit); an idle warp leaves
// after EngineCtl::idle_polls polls, or at once when the host asks, and the
// host launches the kernel again when work comes.
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
__device__ __forceinline__ uint32_t ld_relaxed_sys(volatile const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
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
__device__ __forceinline__ uint32_t engine_pop(const LaunchDesc& L, const EngineCtl& E, Settle& st, bool big) {
  const unsigned long long idx = atomicAdd(big ? L.head_big : L.head, 1ull);
  const unsigned long long lap = (idx >> L.ring_shift) + 1ull;
  const unsigned long long* slot = (big ? L.ready_big : L.ready) + (idx & ((1ull << L.ring_shift) - 1ull));
  uint32_t ns = 32;
  for (uint32_t it = 0;; ++it) {
    const unsigned long long v = ld_acquire64(slot);
    if ((v >> 32) == lap) return (uint32_t)v;
    settle(E, st);
    if ((it & 7u) == 7u && ld_relaxed_sys(E.hstop) != 0u) return kPopDone;
    if (it >= kSpinLimit) {
      atomicOr(L.status, kStatusWaitTimeout);
      return 0xffffffffu;
    }
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
  }
}

// After the kernel has left: the next pop of each ring is the next push
// (tickets taken by warps that left unserved are dropped).
__global__ void reset_heads_kernel(LaunchDesc L) {
  *L.head = *L.tail;
  *L.head_big = *L.tail_big;
}

constexpr int kEngineMinBlocks = 3;

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
  for (;;) {
    uint32_t e;
    if (cont >= 0) {
      e = (uint32_t)cont;
    } else {
      if (tid == 0) g16.bc[7] = engine_pop(L, E, st, true);
      __syncthreads();
      e = g16.bc[7];
      if (e != kPopDone && e != 0xffffffffu) {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&L.frames[e >> 24]);
        uint32_t* to = reinterpret_cast<uint32_t*>(&F);
        for (int i = tid; i < (int)(sizeof(FrameDesc) / 4); i += kGroupThreads) to[i] = __ldcg(from + i);
      }
      __syncthreads();
      if (e == kPopDone) break;
    }
    cont = -1;
    if (e == 0xffffffffu) continue;
    const int f = (int)(e >> 24), t = (int)(e & 0xffffffu);
    if (t >= F.ntasks || !group_task_of(L, F, t)) {
      if (tid == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    }
    if (F.bd == 8) engine_group_task<uint8_t>(L, F, f, t, g8, tid, cont);
    else engine_group_task<uint16_t>(L, F, f, t, g16, tid, cont);
    if (tid == 0) {
      settle(E, st);
      st.old = atom_add_release(&E.fdone[f], 1u);  // thread 0 wrote the result itself
      st.f = f;
      st.n = (uint32_t)F.ntasks;
      st.gen = F.gen;
    }
  }
  if (tid == 0) settle(E, st);
  __syncthreads();
  if (tid < 5) atomicAdd(&L.counters[tid], g16.cnt[tid]);
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32, kEngineMinBlocks) engine_kernel(LaunchDesc L, EngineCtl E) {
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
  for (;;) {
    uint32_t e;
    if (cont >= 0) {
      e = (uint32_t)cont;  // a task of the same frame: its descriptor is here already
    } else {
      e = 0;
      if (lane == 0) e = engine_pop(L, E, st, false);
      e = __shfl_sync(kFull, e, 0);
      if (e == kPopDone) break;
      if (e != 0xffffffffu) {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&L.frames[e >> 24]);
        uint32_t* to = reinterpret_cast<uint32_t*>(&F);
        for (int i = lane; i < (int)(sizeof(FrameDesc) / 4); i += 32) to[i] = __ldcg(from + i);
      }
    }
    __syncwarp();
    cont = -1;
    if (e == 0xffffffffu) continue;
    const int f = (int)(e >> 24), t = (int)(e & 0xffffffu);
    if (t >= F.ntasks || F.mode != RME_PRED_STANDALONE) {
      if (lane == 0) atomicOr(L.status, kStatusBadTask);
      continue;
    }
    if (F.codec == RME_CODEC_HEVC)
      cont = F.bd == 8 ? hevc_task<uint8_t, true>(L, F, f, t, sm8, lane) : hevc_task<uint16_t, true>(L, F, f, t, sm16, lane);
    else
      cont = F.bd == 8 ? h264_task<uint8_t>(L, F, f, t, sm8, lane) : h264_task<uint16_t>(L, F, f, t, sm16, lane);
    if (lane == 0) {
      settle(E, st);
      // Release: lane 0 wrote the task's result itself.
      st.old = atom_add_release(&E.fdone[f], 1u);
      st.f = f;
      st.n = (uint32_t)F.ntasks;
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
  for (int i = threadIdx.x; i < n; i += blockDim.x) push_ready(L, f, (int)roots[i], group_task_of(L, F, (int)roots[i]));
}

// A frame's dependency counts from its shape's template into its slot, and
// its finished-task count cleared: a kernel (beside the resident one)
// rather than a device copy and a memset, which the driver may run as
// kernels of its own that would wait for the resident kernel to leave.
__global__ void prepare_kernel(int32_t* pending, const int32_t* tmpl, int n, uint32_t* fdone) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = i; k < n; k += gridDim.x * blockDim.x) pending[k] = tmpl[k];
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

static cudaError_t launch_prepare(int32_t* pending, const int32_t* tmpl, int n, uint32_t* fdone, cudaStream_t s) {
  prefer_max_shared(prepare_kernel);
  prepare_kernel<<<std::min(64, (n + 255) / 256 + 1), 256, 0, s>>>(pending, tmpl, n, fdone);
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
              kHdrTailBig = 10, kHdrWords = 16;
}  // namespace

struct EngineSlot {
  bool busy = false;
  uint32_t gen = 0;
  int ntasks = 0;
  rme_result* d_out = nullptr;
  size_t out_cap = 0;
  int32_t* d_pending = nullptr;
  size_t pend_cap = 0;
};

struct Engine {
  void* ctx = nullptr;
  int device = 0, grid = 0;
  unsigned long long* d_hdr = nullptr;
  unsigned long long* d_ring = nullptr;  // the warps' ring, then the CTAs' ring
  FrameDesc* d_frames = nullptr;
  FrameDesc* h_frames = nullptr;  // pinned: each slot's descriptor, copied at submit
  uint32_t* d_fdone = nullptr;
  uint32_t* h_flags = nullptr;    // mapped pinned: per slot, the generation finished; then the stop word
  uint32_t* h_stop = nullptr;
  uint32_t* dh_flags = nullptr;   // their device addresses
  uint32_t* dh_stop = nullptr;
  cudaStream_t kstream = nullptr;
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
  if (g->h_stop) {
    *(volatile uint32_t*)g->h_stop = 1u;  // the warps leave (waiting ones within microseconds)
    if (g->launched) cudaEventSynchronize(g->ended);
  }
  cudaDeviceSynchronize();
  for (auto& s : g->slots) {
    if (s.d_out) cudaFree(s.d_out);
    if (s.d_pending) cudaFree(s.d_pending);
  }
  for (void* p : g->outgrown) cudaFree(p);
  if (g->d_hdr) cudaFree(g->d_hdr);
  if (g->d_ring) cudaFree(g->d_ring);
  if (g->d_frames) cudaFree(g->d_frames);
  if (g->h_frames) cudaFreeHost(g->h_frames);
  if (g->d_fdone) cudaFree(g->d_fdone);
  if (g->h_flags) cudaFreeHost(g->h_flags);
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
  if (e == cudaSuccess) e = cudaHostAlloc(&g->h_flags, sizeof(uint32_t) * (kEngineFrames + 32), cudaHostAllocMapped);
  if (e == cudaSuccess) {
    std::memset(g->h_flags, 0, sizeof(uint32_t) * (kEngineFrames + 32));
    g->h_stop = g->h_flags + kEngineFrames;
    e = cudaHostGetDevicePointer((void**)&g->dh_flags, g->h_flags, 0);
  }
  if (e == cudaSuccess) g->dh_stop = g->dh_flags + kEngineFrames;
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
  // A quarter of them run the 32x32 and 64x64 HEVC blocks, a CTA per block.
  const int groups = std::max(1, g->grid / 4);
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
  E.hstop = g->dh_stop;
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
  const int k = g->free_slots.back();
  EngineSlot& s = g->slots[k];
  if (s.out_cap < (size_t)ntasks) {
    if (s.d_out) g->outgrown.push_back(s.d_out);
    s.d_out = nullptr;
    s.out_cap = 0;
    if (cudaMalloc(&s.d_out, sizeof(rme_result) * ntasks) != cudaSuccess) return RME_ENOMEM;
    s.out_cap = ntasks;
  }
  if (s.pend_cap < (size_t)ntasks) {
    if (s.d_pending) g->outgrown.push_back(s.d_pending);
    s.d_pending = nullptr;
    s.pend_cap = 0;
    if (cudaMalloc(&s.d_pending, sizeof(int32_t) * ntasks) != cudaSuccess) return RME_ENOMEM;
    s.pend_cap = ntasks;
  }
  if (++s.gen == 0) s.gen = 1;
  fd.out = s.d_out;
  fd.pending = s.d_pending;
  fd.gen = s.gen;
  g->h_frames[k] = fd;
  if (launch_prepare(s.d_pending, tmpl, ntasks, g->d_fdone + k, upload) != cudaSuccess ||
      cudaMemcpyAsync(g->d_frames + k, g->h_frames + k, sizeof(FrameDesc), cudaMemcpyHostToDevice, upload) !=
          cudaSuccess ||
      launch_publish(g->L, k, roots, nroots, upload) != cudaSuccess)
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
  *(volatile uint32_t*)g->h_stop = 1u;
  cudaError_t e = cudaEventSynchronize(g->ended);
  if (e == cudaSuccess) {
    prefer_max_shared(reset_heads_kernel);
    reset_heads_kernel<<<1, 1, 0, g->kstream>>>(g->L);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->kstream);
  *(volatile uint32_t*)g->h_stop = 0u;
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
