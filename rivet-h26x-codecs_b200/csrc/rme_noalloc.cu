// rme_search_given_noalloc: the GIVEN-mode search for callers that cannot
// allocate device memory.
//
// Some callers of a motion search run where a cudaMalloc is not allowed or
// not possible: an encoder plugin handed a fixed device-memory budget by the
// media pipeline that owns the GPU, code that runs while another component
// holds the allocator, or a latency-critical loop where the device-wide
// synchronisation of cudaMalloc/cudaFree is unacceptable. They hold their
// pictures and buffers already; this entry point searches their jobs over
// their planes and writes their output buffer, and keeps everything else it
// needs — the frame descriptor, the launch's queue header and slots, the
// H.264 rate table — in one file-scope device array of fixed size.
//
// That array is in every process that loads the library, on every device
// it is used on, until exit. Its address is looked up once per device
// (cudaGetSymbolAddress, with that device current) on the first call there,
// so that first call should come before any stream capture. All calls
// share the array: calls whose work overlaps on a GPU (two host threads,
// or two streams) race on it, and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "rme_internal.h"

namespace rme {
namespace {

constexpr int kNoAllocMaxJobs = 65536;
constexpr size_t kOffFrame = 0;     // FrameDesc
constexpr size_t kOffMisc = 512;    // 16 x u64: queue header, counters, status, epoch
constexpr size_t kOffTab = 1024;    // H.264 MvCostTable (8193 x u16)
constexpr size_t kOffSlots = 17664; // queue slots (kNoAllocMaxJobs x u64)
constexpr size_t kScratchBytes = kOffSlots + (size_t)kNoAllocMaxJobs * 8;
static_assert(sizeof(FrameDesc) <= kOffMisc - kOffFrame, "frame descriptor outgrew its scratch slot");
static_assert(kOffTab + kMvTab * sizeof(uint16_t) <= kOffSlots, "rate table outgrew its scratch slot");
static_assert(kScratchBytes == 541952, "the documented scratch size");

// The scratch: 541,952 bytes (about 529 KiB). Device code could name it
// directly; host code must use the address cudaGetSymbolAddress returns,
// never the symbol.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

__global__ void fill_ready(unsigned long long* slots, int n, uint32_t epoch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) slots[i] = ((unsigned long long)epoch << 32) | (uint32_t)i;
}

struct DeviceScratch {
  unsigned char* base = nullptr;
  uint32_t epoch = 0;
};
std::mutex g_mu;
DeviceScratch g_dev[64];

bool plane_ok(const rme_plane_set& ps, int need_pad, int cw, int ch) {
  return ps.base && ps.pad >= need_pad && ps.stride >= cw + 2 * ps.pad &&
         ps.plane_elems >= (int64_t)ps.stride * (ch + 2 * ps.pad) && (reinterpret_cast<uintptr_t>(ps.base) & 15) == 0;
}

}  // namespace
}  // namespace rme

using namespace rme;

extern "C" int rme_search_given_noalloc(const rme_picture_desc* d, const rme_params* p, const rme_plane_set* src,
                                        const rme_plane_set* refs, int32_t nref, const rme_job* jobs, int32_t njobs,
                                        rme_result* out, void* stream) {
  if (!d || !p || !src || !refs || !jobs || !out) return RME_EINVAL;
  if (d->codec != RME_CODEC_H264 && d->codec != RME_CODEC_HEVC) return RME_EINVAL;
  if (d->bit_depth < 8 || d->bit_depth > 12 || d->width < 16 || d->height < 16) return RME_EINVAL;
  if (p->codec != d->codec || p->predictor_mode != RME_PRED_GIVEN) return RME_EINVAL;
  if (param_error(p, *d)) return RME_EINVAL;  // the limits every other search entry point applies
  if (nref < 1 || nref > RME_MAX_REFS) return RME_EINVAL;
  if (njobs < 0 || njobs > kNoAllocMaxJobs) return RME_EINVAL;  // beyond the scratch's queue
  if (njobs == 0) return RME_OK;
  const bool h264 = d->codec == RME_CODEC_H264;
  const int cw = h264 ? (d->width + 15) / 16 * 16 : d->width, ch = h264 ? (d->height + 15) / 16 * 16 : d->height;
  const int pad = h264 ? p->h264_pad : p->hevc_pad;
  if (!plane_ok(*src, pad, cw, ch)) return RME_EINVAL;
  for (int r = 0; r < nref; ++r)
    if (!plane_ok(refs[r], pad, cw, ch)) return RME_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return RME_ECUDA;
  unsigned char* base;
  uint32_t epoch;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceScratch& ds = g_dev[dev];
    if (!ds.base) {
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return RME_ECUDA;
      ds.base = (unsigned char*)ptr;
    }
    if (++ds.epoch == 0) ds.epoch = 1;  // slots of an earlier call never match
    base = ds.base;
    epoch = ds.epoch;
  }

  // The frame descriptor: the caller's planes, jobs and output buffer.
  FrameDesc fd;
  std::memset(&fd, 0, sizeof(fd));
  auto planes = [](const rme_plane_set& ps) {
    DevPlanes dp;
    dp.base = ps.base;
    dp.plane_elems = ps.plane_elems;
    dp.stride = ps.stride;
    dp.origin = ps.pad * ps.stride + ps.pad;
    return dp;
  };
  fd.codec = d->codec;
  fd.bd = d->bit_depth;
  fd.mode = RME_PRED_GIVEN;
  fd.nref = nref;
  fd.width = cw;
  fd.height = ch;
  fd.pad = pad;
  fd.src = planes(*src);
  for (int r = 0; r < nref; ++r) fd.ref[r] = planes(refs[r]);
  fd.jobs = jobs;
  fd.out = out;
  fd.pending = nullptr;
  fd.ntasks = njobs;
  static thread_local uint16_t tab[kMvTab];
  if (h264) {
    h264_cost_table(h264_lambda_satd(p->qp), tab);
    fd.tab = reinterpret_cast<const uint16_t*>(base + kOffTab);
    fd.range = p->h264_range;
    fd.hpel_iters = p->h264_hpel_iters;
    fd.qpel_iters = p->h264_qpel_iters;
    fd.umh = p->h264_umh;
    fd.qpel_diamond = p->h264_qpel_diamond;
    fd.dia = p->h264_dia;
    fd.vr = p->h264_vertical_range;
    fd.refine_ratio = p->h264_refine_ratio;
  } else {
    fd.lam = hevc_lambda(p->qp, d->bit_depth, p->hevc_lambda_scale);
    fd.search_range = p->hevc_search_range;
    fd.search_rings = p->hevc_search_rings;
    fd.quarter_cross = p->hevc_quarter_cross;
  }

  // The queue header starts at zero but for the tail (every job is ready)
  // and this call's epoch; the slots are written by a kernel.
  unsigned long long misc[16];
  std::memset(misc, 0, sizeof(misc));
  misc[1] = (unsigned long long)njobs;
  misc[10] = epoch;
  unsigned long long* d_misc = reinterpret_cast<unsigned long long*>(base + kOffMisc);
  unsigned long long* slots = reinterpret_cast<unsigned long long*>(base + kOffSlots);
  if (cudaMemcpyAsync(base + kOffFrame, &fd, sizeof(fd), cudaMemcpyHostToDevice, s) != cudaSuccess) return RME_ECUDA;
  if (cudaMemcpyAsync(d_misc, misc, sizeof(misc), cudaMemcpyHostToDevice, s) != cudaSuccess) return RME_ECUDA;
  if (h264 && cudaMemcpyAsync(base + kOffTab, tab, sizeof(tab), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return RME_ECUDA;
  fill_ready<<<(njobs + 255) / 256, 256, 0, s>>>(slots, njobs, epoch);
  if (cudaGetLastError() != cudaSuccess) return RME_ECUDA;

  LaunchDesc L = {};
  L.frames = reinterpret_cast<const FrameDesc*>(base + kOffFrame);
  L.ready = slots;
  L.total = njobs;
  L.head = d_misc;
  L.tail = d_misc + 1;
  L.counters = d_misc + 4;
  L.status = reinterpret_cast<uint32_t*>(d_misc + 9);
  L.epoch = reinterpret_cast<const uint32_t*>(d_misc + 10);
  L.done = nullptr;  // GIVEN jobs only: no task makes another ready
  const int bytes = d->bit_depth == 8 ? 1 : 2;
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return RME_ECUDA;
  const int64_t want = ((int64_t)njobs + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)nsm * search_blocks_per_sm(bytes, d->codec, kDefaultVariant), want));
  if (launch_search(L, bytes, d->codec, kDefaultVariant, grid, s) != cudaSuccess) return RME_ECUDA;
  if (cudaMemcpyAsync(misc, d_misc, sizeof(misc), cudaMemcpyDeviceToHost, s) != cudaSuccess) return RME_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return RME_ECUDA;
  if ((uint32_t)misc[9] != 0 || misc[4] != (unsigned long long)njobs) return RME_EDEVICE;
  return RME_OK;
}
