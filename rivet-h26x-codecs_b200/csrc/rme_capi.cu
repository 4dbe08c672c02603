// Host side of librivet_me.so: the C ABI of include/rivet_me.h.
//
// A context owns device pictures (padded planes built on upload), the cost
// tables per (codec, QP, depth, multiplier), the task orders per frame
// shape, and the launch buffers. A frame search (or a batch of frames) is:
// frame descriptors + the work queue to the device, one persistent search
// launch, results back. Host code here only prepares and moves data; every
// candidate is scored on the device.
//
// The Lagrangian tables are computed in f32 exactly as the reference does
// (this file is compiled with -ffp-contract=off): H.264 MvCostTable::new
// (h264_hpel.rs:453-459) at lambda_satd (h264_analyse.rs:402-404); HEVC
// (lam * bits as f32) as u32 (h265_me.rs:3776, 3890) at lambda * 2^(bd-8)
// (h265_intra.rs:1141-2013).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "rme_internal.h"

namespace rme {

// ---- Lagrangian tables -------------------------------------------------------
float h264_mvd_bits(int d) {  // h264_hpel.rs:407-429
  uint32_t a = (uint32_t)std::abs(d);
  if (a == 0) return 1.0f;
  float prefix = (float)std::min(a, 9u);
  float bits = 1.0f + 0.85f * prefix;
  if (a < 9) {
    bits += 0.85f;
  } else {
    uint32_t v = a - 9, k = 3;
    while (v >= (1u << k)) {
      v -= 1u << k;
      k += 1;
    }
    bits += (float)(k - 3 + 1 + k);
  }
  return bits + 1.0f;
}
float h264_lambda_satd(int qp) { return std::sqrt(0.85f * std::exp2((float)(qp - 12) / 3.0f)); }
float hevc_lambda(int qp, int bd, float scale) {
  float base = 0.85f * std::exp2((float)(qp - 12) / 3.0f) * scale;
  return std::sqrt(base) * (float)(1u << (bd - 8));
}
void h264_cost_table(float lam, uint16_t* tab) {  // MvCostTable::new (h264_hpel.rs:453-459)
  for (int d = -kMvSpan; d <= kMvSpan; ++d) tab[d + kMvSpan] = (uint16_t)std::min(lam * h264_mvd_bits(d) + 0.5f, 65535.0f);
}

const char* param_error(const rme_params* p, const rme_picture_desc& d) {
  if (!p) return "null params";
  if (p->codec != d.codec) return "params codec differs from the picture's";
  if (p->predictor_mode != RME_PRED_GIVEN && p->predictor_mode != RME_PRED_STANDALONE) return "bad predictor_mode";
  if (p->qp < -12 || p->qp > 63) return "qp out of range";
  if (d.codec == RME_CODEC_H264) {
    if (p->h264_pad < 8 || p->h264_pad > kH264Pad) return "h264_pad must be 8..32";
    if (p->h264_range < 0 || p->h264_range > 512 || p->h264_hpel_iters < 0 || p->h264_qpel_iters < 0 ||
        p->h264_hpel_iters > 64 || p->h264_qpel_iters > 64)
      return "bad H.264 MeCfg";
    // vertical_search is range - 1 of a level's MaxVmvR >= 0: at least -1.
    // (A window emptied by it still clamps every point inside the plane.)
    if (p->h264_vertical_range < -1) return "h264_vertical_range below -1";
    if (!std::isfinite(p->h264_refine_ratio)) return "h264_refine_ratio must be finite";
  } else {
    if (p->hevc_pad < 8 || p->hevc_pad > kHevcPad) return "hevc_pad must be 8..80";
    if (p->hevc_search_range < 0 || p->hevc_search_range > 1024 || p->hevc_search_rings < 0 ||
        p->hevc_search_rings > 64)
      return "bad HEVC search settings";
    // Tune::lambda_of's multipliers are small positive numbers; a scale
    // outside [0, 1024] (or not a number) has no finite per-bit price.
    if (!(p->hevc_lambda_scale >= 0.0f && p->hevc_lambda_scale <= 1024.0f)) return "hevc_lambda_scale must be 0..1024";
    if (p->predictor_mode == RME_PRED_STANDALONE && ((p->hevc_pu_mask & 0xF) == 0 || (p->hevc_pu_mask & ~0xF)))
      return "hevc_pu_mask must select sizes among 8..64";
    if (p->hevc_amp & ~0xF) return "hevc_amp selects among four AMP modes";
  }
  return nullptr;
}

}  // namespace rme

using namespace rme;

namespace {

// A launch's tasks split into parts by kind, one search kernel each:
// part = 2 * (deeper than 8 bits) + (H.264).
constexpr int kParts = 4;
// The launch header in device memory (u64 words): head and tail of each
// part's queue, then the counters, the status word and the epoch.
// The launch header: head and tail of each part's queue (0..7), the
// counters (8..12), status, epoch, then each part's finished-task count.
constexpr int64_t kSpecTasks = 200000;  // about two 1080p frames of 2Nx2N PUs, 2 references
constexpr int kMiscCounters = 8, kMiscStatus = 13, kMiscEpoch = 14, kMiscDone = 16, kMiscBig = 20, kMiscWords = 32;

int part_of(const FrameDesc& fd) { return 2 * (fd.bd > 8) + (fd.codec == RME_CODEC_H264); }
int part_bytes(int k) { return k >= 2 ? 2 : 1; }
int part_codec(int k) { return (k & 1) ? RME_CODEC_H264 : RME_CODEC_HEVC; }

uint32_t h264_ref_bits_cost(float lam1, int r, int nref) {  // h264_analyse.rs:1934-1942
  float bits = nref == 1 ? 0.0f : nref == 2 ? 1.0f : (float)(2 * (32 - __builtin_clz((unsigned)(r + 1))) - 1);
  return (uint32_t)(lam1 * bits);
}
uint32_t hevc_ref_idx_bits(int r, int nref) {
  if (nref <= 1) return 0;
  return r < nref - 1 ? (uint32_t)(r + 1) : (uint32_t)r;
}

// Buffers that grow on demand. `generation` counts reallocations across all
// of them, so launch graphs captured over an old buffer are never replayed.
static uint64_t g_buffer_generation = 0;

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t want) {
    if (want <= n) return cudaSuccess;
    ++g_buffer_generation;
    const size_t grow = std::max(want, n * 3 / 2);  // geometric: few reallocations
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, grow * sizeof(T) + 64);
    if (e == cudaSuccess) n = grow;
    return e;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
template <class T>
struct PinBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t want) {
    if (want <= n) return cudaSuccess;
    ++g_buffer_generation;
    const size_t grow = std::max(want, n * 3 / 2);
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMallocHost(&p, grow * sizeof(T) + 64);
    if (e == cudaSuccess) n = grow;
    return e;
  }
  ~PinBuf() {
    if (p) cudaFreeHost(p);
  }
};

struct Picture {
  rme_picture_desc d{};
  int cw = 0, ch = 0, pad = 0, nplanes = 0;
  void* buf = nullptr;
  size_t bytes = 0;
  DevPlanes planes{};
  bool is_ref = false;
  void* chroma = nullptr;  // cb then cr, unpadded (cw/2 x ch/2), packed
  size_t chroma_bytes = 0;
  void* lowres = nullptr;  // the lookahead's half-resolution plane, then its intra costs
  LowresDesc lr{};
  ~Picture() {
    if (buf) cudaFree(buf);
    if (chroma) cudaFree(chroma);
    if (lowres) cudaFree(lowres);
  }
};

struct Tables {
  uint16_t* tab = nullptr;  // H.264 MvCostTable
  float lam = 0.0f;         // the Lagrangian (H.264 lambda_satd; HEVC lam)
};

struct Deps {  // the dependency structure of one frame shape
  int32_t* pending = nullptr;    // device: per task, how many tasks it reads
  std::vector<uint32_t> ready;   // tasks that read none, in order
  uint32_t* d_ready = nullptr;   // device copy of `ready` (the resident engine publishes from it)
  size_t ntasks = 0;
  // The row form (HEVC without AMP): the rows a warp runs (16x16 and 8x8)
  // and the rows a CTA runs (64x64 and 32x32), as row_entry words, each
  // list ordered by the row's first sample row, larger blocks first: every
  // row comes after the rows it reads (its upper row, its parents' rows).
  std::vector<uint32_t> rows, rows_big;
  uint32_t* d_rows = nullptr;    // device: rows, then rows_big
};

struct Graph {
  cudaGraphExec_t exec = nullptr;
  int seen = 0;  // launches of this shape so far: captured on the second
};

// A launch shape the tuner chooses among: the search kernel's occupancy
// variant (registers per thread against resident warps), in the latency form
// the share of CTAs that search 32x32 and 64x64 HEVC blocks a CTA per block
// (0, a quarter or half of the SMs), and whether 8x8 blocks refine from
// staged phase patches (the search window's neighbourhood in shared memory)
// or straight from the caches; and whether HEVC STANDALONE frames without
// AMP run in the row form (a warp or a CTA per row of blocks; `groups` 3:
// a CTA for every row of large blocks, up to half the grid).
struct Shape {
  int variant, groups, patch, rows;
};
constexpr Shape kThroughputShapes[] = {{1, 0, 0, 0}, {0, 0, 0, 0}, {2, 0, 0, 0}};
constexpr Shape kLatencyHevcShapes[] = {{0, 3, 0, 1}, {0, 3, 1, 1}, {1, 3, 0, 1}, {1, 2, 1, 0},
                                        {1, 2, 0, 0}, {1, 1, 1, 0}, {1, 0, 0, 0}, {0, 2, 1, 0}};
constexpr Shape kLatencyShapes[] = {{1, 0, 0, 0}, {0, 0, 0, 0}, {2, 0, 0, 0}};
constexpr int kTuneRounds = 2;  // timings per shape before the tuner chooses (launch times vary)
constexpr int kNumShapes[3] = {(int)(sizeof(kThroughputShapes) / sizeof(Shape)),
                               (int)(sizeof(kLatencyHevcShapes) / sizeof(Shape)),
                               (int)(sizeof(kLatencyShapes) / sizeof(Shape))};

// One search launch's buffers and events. A context keeps kSlots of them and
// takes them in turn: a synchronous search finishes its launch before it
// returns; an asynchronous one leaves it in flight on the caller's stream
// until rme_sync (or until its slot comes round again, which waits for it).
constexpr int kSlots = 4;
struct Slot {
  DevBuf<FrameDesc> d_frames;
  DevBuf<unsigned long long> d_ready;  // the dataflow queue's slots
  DevBuf<rme_result> d_out;
  DevBuf<int32_t> d_pending;
  DevBuf<rme_job> d_jobs;
  DevBuf<unsigned long long> d_misc;  // the launch header (kMisc*)
  DevBuf<unsigned long long> d_mvf;   // the row form's published vectors (tagged with the epoch)
  PinBuf<FrameDesc> h_frames;
  PinBuf<rme_result> h_out;
  PinBuf<unsigned long long> h_misc;
  PinBuf<unsigned long long> h_init;  // [misc header | initial queue entries]
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;
  uint32_t epoch = 0;
  // The launch in flight: its stream, its task count, the tuner class it
  // times, and (synchronous calls into pageable memory) where its results go.
  bool busy = false;
  cudaStream_t stream = nullptr;
  int64_t total = 0;
  void* tuning = nullptr;
  int tune_shapes = 0;
  rme_result* host_out = nullptr;
  std::vector<int64_t> host_off, host_count, dev_off;
  ~Slot() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (done) cudaEventDestroy(done);
  }
};

struct Ctx {
  int device = 0, nsm = 0;
  int bps[kParts][kSearchVariants][2] = {};  // resident search blocks per SM, per part, variant, form
  // The tuner: per (part, form, log2 of its task count), each launch shape
  // of that class (kShapes) is timed on one real launch, then the fastest is
  // kept. Results do not depend on the shape.
  struct Tune {
    int best = -1, tried = 0;
    float ms[8] = {};  // per shape, its best time so far
  };
  std::map<std::pair<int, int>, Tune> tune;
  bool tune_on = true;
  cudaStream_t stream = nullptr;
  // The parts of a launch after the first run on streams of their own,
  // forked from and joined back to the caller's stream.
  cudaStream_t aux[kParts] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[kParts] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t evp0 = nullptr, evp1 = nullptr;
  std::map<int, std::unique_ptr<Picture>> pics;
  std::map<std::tuple<int, int, int, uint32_t>, Tables> tables;
  std::map<std::vector<int64_t>, Deps> deps;
  std::string err;
  rme_stats last{};
  // launch buffers, taken in turn
  Slot slots[kSlots];
  int next_slot = 0;
  // Errors of asynchronous launches finished before their rme_sync (their
  // slot was needed again), per stream: the first error code, the device
  // status bits.
  std::map<cudaStream_t, std::pair<int, uint32_t>> async_err;
  DevBuf<int32_t> d_lorder;           // lookahead: claim order (per block shape), done flags, results
  std::pair<int, int> lorder_shape{0, 0};
  DevBuf<int32_t> d_ldone;
  DevBuf<uint32_t> d_lcost, d_lsad;
  DevBuf<rme_mv> d_lmv, d_lmv2;
  DevBuf<LowresDesc> d_lpairs;
  DevBuf<unsigned long long> d_wp;    // weighted prediction: moments, weighted SAD
  DevBuf<rme_bi_job> d_bijobs;        // bi-prediction: jobs, SATDs, refine_bi targets
  DevBuf<uint32_t> d_bisatd;
  DevBuf<uint8_t> d_bitarget;
  DevBuf<rme_job> d_wjobs;            // HEVC weighted refinement: jobs, results
  DevBuf<rme_result> d_wout;
  DevBuf<rme_h264_bi_job> d_h264bi;   // H.264 B pairs: jobs, refined vectors
  DevBuf<rme_mv> d_bimv;
  DevBuf<int32_t> d_cblk;             // chroma: blocks, vectors, output offsets, output
  DevBuf<rme_mv> d_cmv;
  DevBuf<int64_t> d_coff;
  DevBuf<uint8_t> d_cout;
  std::map<std::vector<int64_t>, Graph> graphs;
  bool planes_pending = false;  // uploads recorded between evp0 and evp1 since the last search
  ~Ctx() {
    for (auto& g : graphs)
      if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
    for (auto& d : deps) {
      if (d.second.pending) cudaFree(d.second.pending);
      if (d.second.d_ready) cudaFree(d.second.d_ready);
      if (d.second.d_rows) cudaFree(d.second.d_rows);
    }
    for (auto& t : tables)
      if (t.second.tab) cudaFree(t.second.tab);
    if (evp0) cudaEventDestroy(evp0);
    if (evp1) cudaEventDestroy(evp1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (int k = 0; k < kParts; ++k) {
      if (ev_join[k]) cudaEventDestroy(ev_join[k]);
      if (aux[k]) cudaStreamDestroy(aux[k]);
    }
    if (stream) cudaStreamDestroy(stream);
  }
};

int fail(Ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
int cuda_fail(Ctx* c, cudaError_t e, const char* what) {
  return fail(c, RME_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                         \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
  } while (0)

bool valid_desc(const rme_picture_desc* d) {
  return d && (d->codec == RME_CODEC_H264 || d->codec == RME_CODEC_HEVC) && d->bit_depth >= 8 &&
         d->bit_depth <= 12 && d->width >= 16 && d->height >= 16 && d->stride >= d->width &&
         d->width <= 8192 && d->height <= 4352;
}

int level_sizes(const rme_params* p, int* sizes) {
  int n = 0;
  for (int k = 3; k >= 0; --k)
    if (p->hevc_pu_mask & (1 << k)) sizes[n++] = 8 << k;
  return n;
}

// The two units of an asymmetric partition of the N x N CU at (x, y): mode
// bit 0 2NxnU, 1 2NxnD, 2 nLx2N, 3 nRx2N, part 0 the top/left unit.
void amp_unit(int mode, int part, int x, int y, int N, int32_t* b) {
  const int q = N / 4;
  b[0] = x;
  b[1] = y;
  b[2] = b[3] = N;
  if (mode < 2) {
    b[3] = (part == (mode == 0)) ? 3 * q : q;
    if (part) b[1] = y + (mode == 0 ? q : 3 * q);
  } else {
    b[2] = (part == (mode == 2)) ? 3 * q : q;
    if (part) b[0] = x + (mode == 2 ? q : 3 * q);
  }
}

int count_blocks(const rme_picture_desc* d, const rme_params* p, int32_t* blocks) {
  int n = 0;
  if (d->codec == RME_CODEC_H264) {
    int mbw = (d->width + 15) / 16, mbh = (d->height + 15) / 16;
    for (int my = 0; my < mbh; ++my)
      for (int mx = 0; mx < mbw; ++mx, ++n)
        if (blocks) {
          blocks[4 * n] = mx * 16;
          blocks[4 * n + 1] = my * 16;
          blocks[4 * n + 2] = blocks[4 * n + 3] = 16;
        }
    return n;
  }
  int sizes[4], nl = level_sizes(p, sizes);
  for (int l = 0; l < nl; ++l) {
    int N = sizes[l];
    for (int by = 0; by + N <= d->height; by += N)
      for (int bx = 0; bx + N <= d->width; bx += N, ++n)
        if (blocks) {
          blocks[4 * n] = bx;
          blocks[4 * n + 1] = by;
          blocks[4 * n + 2] = blocks[4 * n + 3] = N;
        }
  }
  // AMP units: per level of 16 or more, per CU, per enabled mode, two units.
  if (p->predictor_mode == RME_PRED_STANDALONE)
    for (int l = 0; l < nl && sizes[l] >= 16; ++l) {
      int N = sizes[l];
      for (int by = 0; by + N <= d->height; by += N)
        for (int bx = 0; bx + N <= d->width; bx += N)
          for (int m = 0; m < 4; ++m)
            if ((p->hevc_amp >> m) & 1)
              for (int k = 0; k < 2; ++k, ++n)
                if (blocks) amp_unit(m, k, bx, by, N, blocks + 4 * n);
    }
  return n;
}

int check_params(Ctx* c, const rme_params* p, const rme_picture_desc& d) {
  const char* why = param_error(p, d);
  return why ? fail(c, RME_EINVAL, why) : 0;
}

const Tables* get_tables(Ctx* c, const rme_params* p, int bd, int* rc) {
  uint32_t scale_bits;
  float scale = p->codec == RME_CODEC_HEVC ? p->hevc_lambda_scale : 1.0f;
  std::memcpy(&scale_bits, &scale, 4);
  auto key = std::make_tuple(p->codec, p->qp, p->codec == RME_CODEC_HEVC ? bd : 8, scale_bits);
  auto it = c->tables.find(key);
  if (it != c->tables.end()) return &it->second;
  Tables t;
  if (p->codec == RME_CODEC_H264) {
    std::vector<uint16_t> tab(kMvTab);
    float lam = h264_lambda_satd(p->qp);
    h264_cost_table(lam, tab.data());
    t.lam = lam;
    cudaError_t e = cudaMalloc(&t.tab, kMvTab * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMemcpy(t.tab, tab.data(), kMvTab * sizeof(uint16_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      *rc = cuda_fail(c, e, "table upload");
      return nullptr;
    }
  } else {
    t.lam = hevc_lambda(p->qp, bd, scale);
  }
  return &(c->tables[key] = t);
}

// The STANDALONE dependency structure of a frame shape: per task how many
// other tasks' results it reads (HEVC: the left and upper blocks of its
// level, the enclosing block of the next larger evaluated size; H.264: the
// A, B, C and D macroblocks), and the tasks that read none. The kernel
// releases exactly these edges (rme_search.cu), so every count reaches zero.
const Deps* get_deps(Ctx* c, const rme_picture_desc& d, const rme_params* p, int nref, int* rc) {
  std::vector<int64_t> sig = {d.codec, d.width, d.height, nref, d.codec == RME_CODEC_HEVC ? p->hevc_pu_mask : 0,
                              d.codec == RME_CODEC_HEVC ? p->hevc_amp : 0};
  auto it = c->deps.find(sig);
  if (it != c->deps.end()) return &it->second;
  std::vector<int32_t> pend;
  Deps dp;
  if (d.codec == RME_CODEC_H264) {
    const int mbw = (d.width + 15) / 16, mbh = (d.height + 15) / 16;
    for (int my = 0; my < mbh; ++my)
      for (int mx = 0; mx < mbw; ++mx)
        pend.push_back((mx > 0) + (my > 0) + (my > 0 && mx + 1 < mbw) + (mx > 0 && my > 0));
  } else {
    int sizes[4];
    const int nl = level_sizes(p, sizes);
    for (int l = 0; l < nl; ++l) {
      const int N = sizes[l], nbx = d.width / N, nby = d.height / N;
      for (int by = 0; by < nby; ++by)
        for (int bx = 0; bx < nbx; ++bx) {
          bool parent = false;
          if (l > 0) {
            const int Np = sizes[l - 1];
            parent = bx * N / Np < d.width / Np && by * N / Np < d.height / Np;
          }
          for (int r = 0; r < nref; ++r) pend.push_back((bx > 0) + (by > 0) + parent);
        }
    }
    // An AMP unit reads its CU's 2Nx2N result.
    const int namp = count_blocks(&d, p, nullptr) - (int)(pend.size() / nref);
    for (int k = 0; k < namp * nref; ++k) pend.push_back(1);
  }
  for (size_t t = 0; t < pend.size(); ++t)
    if (pend[t] == 0) dp.ready.push_back((uint32_t)t);
  dp.ntasks = pend.size();
  if (d.codec == RME_CODEC_HEVC && p->hevc_amp == 0) {
    // Reference-major: a block's warps take consecutive rows of one
    // reference, whose reference bands overlap in the SM's L1.
    struct Row {
      int r, y, size;
      uint32_t entry;
    };
    std::vector<Row> all;
    int sizes[4];
    const int nl = level_sizes(p, sizes);
    for (int l = 0; l < nl; ++l) {
      const int N = sizes[l];
      if (d.width / N == 0) continue;
      for (int row = 0; row < d.height / N; ++row)
        for (int r = 0; r < nref; ++r) all.push_back({r, row * N, N, row_entry(l, r, row)});
    }
    std::stable_sort(all.begin(), all.end(), [](const Row& a, const Row& b) {
      return a.r != b.r ? a.r < b.r : a.y != b.y ? a.y < b.y : a.size > b.size;
    });
    for (const Row& w : all) (w.size >= 32 ? dp.rows_big : dp.rows).push_back(w.entry);
  }
  cudaError_t e = cudaMalloc(&dp.pending, std::max<size_t>(pend.size(), 1) * sizeof(int32_t));
  if (e == cudaSuccess)
    e = cudaMemcpy(dp.pending, pend.data(), pend.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&dp.d_ready, std::max<size_t>(dp.ready.size(), 1) * sizeof(uint32_t));
  if (e == cudaSuccess)
    e = cudaMemcpy(dp.d_ready, dp.ready.data(), dp.ready.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
  const size_t nrows = dp.rows.size() + dp.rows_big.size();
  if (e == cudaSuccess && nrows > 0) e = cudaMalloc(&dp.d_rows, nrows * sizeof(uint32_t));
  if (e == cudaSuccess && !dp.rows.empty())
    e = cudaMemcpy(dp.d_rows, dp.rows.data(), dp.rows.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !dp.rows_big.empty())
    e = cudaMemcpy(dp.d_rows + dp.rows.size(), dp.rows_big.data(), dp.rows_big.size() * sizeof(uint32_t),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (dp.pending) cudaFree(dp.pending);
    if (dp.d_ready) cudaFree(dp.d_ready);
    if (dp.d_rows) cudaFree(dp.d_rows);
    *rc = cuda_fail(c, e, "dependency template");
    return nullptr;
  }
  return &(c->deps[sig] = std::move(dp));
}

int picture_of(Ctx* c, int id, Picture** out) {
  auto it = c->pics.find(id);
  if (it == c->pics.end()) return fail(c, RME_ENOTFOUND, "picture " + std::to_string(id) + " not uploaded");
  *out = it->second.get();
  return 0;
}

// Fill one FrameDesc. `slot_out`/`slot_flags` index the launch buffers.
int make_frame(Ctx* c, const rme_frame* f, const rme_params* p, FrameDesc* fd, rme_result* dout, int32_t* dflags,
               const rme_job* djobs, int* ntasks) {
  Picture* src;
  int rc = picture_of(c, f->src_id, &src);
  if (rc) return rc;
  if (f->nref < 1 || f->nref > RME_MAX_REFS) return fail(c, RME_EINVAL, "nref must be 1..4");
  if ((rc = check_params(c, p, src->d))) return rc;
  std::memset(fd, 0, sizeof(*fd));
  fd->codec = src->d.codec;
  fd->bd = src->d.bit_depth;
  fd->mode = p->predictor_mode;
  fd->nref = f->nref;
  fd->width = src->cw;
  fd->height = src->ch;
  fd->src = src->planes;
  for (int r = 0; r < f->nref; ++r) {
    Picture* rp;
    if ((rc = picture_of(c, f->ref_ids[r], &rp))) return rc;
    if (!rp->is_ref) return fail(c, RME_EINVAL, "reference picture was uploaded without as_ref");
    if (rp->d.codec != src->d.codec || rp->d.bit_depth != src->d.bit_depth || rp->d.width != src->d.width ||
        rp->d.height != src->d.height)
      return fail(c, RME_EINVAL, "reference format differs from the source's");
    fd->ref[r] = rp->planes;
  }
  const Tables* t = get_tables(c, p, src->d.bit_depth, &rc);
  if (!t) return rc;
  if (fd->codec == RME_CODEC_HEVC) {
    fd->pad = p->hevc_pad;
    fd->search_range = p->hevc_search_range;
    fd->search_rings = p->hevc_search_rings;
    fd->quarter_cross = p->hevc_quarter_cross;
    fd->lam = t->lam;
    int sizes[4];
    fd->nlevels = level_sizes(p, sizes);
    for (int l = 0; l < fd->nlevels; ++l) {
      fd->size[l] = sizes[l];
      fd->nbx[l] = src->d.width / sizes[l];
      fd->nby[l] = src->d.height / sizes[l];
      fd->base[l + 1] = fd->base[l] + fd->nbx[l] * fd->nby[l];
    }
    // Blocks of 32 or more (the first levels): the tasks a CTA runs in the
    // latency form.
    if (p->predictor_mode == RME_PRED_STANDALONE) {
      int lb = 0;
      while (lb < fd->nlevels && fd->size[lb] >= 32) ++lb;
      fd->big_end = fd->base[lb];
    }
    if (p->predictor_mode == RME_PRED_STANDALONE && p->hevc_amp) {
      fd->amp = p->hevc_amp;
      fd->amp_nmodes = __builtin_popcount((unsigned)p->hevc_amp);
      fd->amp_base[0] = fd->base[fd->nlevels];
      while (fd->amp_nlev < fd->nlevels && fd->size[fd->amp_nlev] >= 16) {
        const int l = fd->amp_nlev++;
        fd->amp_base[l + 1] = fd->amp_base[l] + fd->nbx[l] * fd->nby[l] * 2 * fd->amp_nmodes;
      }
    }
  } else {
    fd->pad = p->h264_pad;
    fd->tab = t->tab;
    fd->range = p->h264_range;
    fd->hpel_iters = p->h264_hpel_iters;
    fd->qpel_iters = p->h264_qpel_iters;
    fd->umh = p->h264_umh;
    fd->qpel_diamond = p->h264_qpel_diamond;
    fd->dia = p->h264_dia;
    fd->vr = p->h264_vertical_range;
    fd->refine_ratio = p->h264_refine_ratio;
    for (int r = 0; r < f->nref; ++r) fd->ref_cost[r] = h264_ref_bits_cost(t->lam, r, f->nref);
  }
  if (p->predictor_mode == RME_PRED_GIVEN) {
    if (f->njobs < 0 || (f->njobs > 0 && !f->jobs)) return fail(c, RME_EINVAL, "jobs missing");
    for (int j = 0; j < f->njobs; ++j) {
      const rme_job& jb = f->jobs[j];
      if (jb.ref < 0 || jb.ref >= f->nref || jb.nseeds < 0 || jb.nseeds > RME_MAX_SEEDS || jb.w < 4 || jb.h < 4 ||
          jb.w > 64 || jb.h > 64 || (jb.w & 3) || (jb.h & 3) || jb.x < 0 || jb.y < 0 || jb.x + jb.w > src->cw ||
          jb.y + jb.h > src->ch)
        return fail(c, RME_EINVAL, "job " + std::to_string(j) + " out of range");
      if (fd->codec == RME_CODEC_H264 && jb.nseeds > 8)
        return fail(c, RME_EINVAL, "H.264 jobs take at most 8 candidates (p_mb's cands)");
    }
    fd->jobs = djobs;
    *ntasks = f->njobs;
  } else {
    int nb = count_blocks(&src->d, p, nullptr);
    *ntasks = fd->codec == RME_CODEC_H264 ? nb : nb * f->nref;
  }
  fd->out = dout;
  fd->pending = dflags;
  fd->ntasks = *ntasks;
  return 0;
}

// Finish the launch in flight on slot `sl`: wait for it, check the device
// status and the task count, keep its statistics (and feed the tuner), move
// results bound for pageable memory. Returns 0 or an error code.
// `wait_planes`: a synchronous call waits for the uploads since the previous
// search to report their device time; an asynchronous launch's completion
// (rme_sync, or its slot taken again) reports it only if they are done, so
// that it never waits on uploads queued after the launch.
int finish_launch(Ctx* c, Slot& sl, bool wait_planes = true) {
  if (!sl.busy) return 0;
  sl.busy = false;
  CK(cudaEventSynchronize(sl.done));
  const uint32_t status = (uint32_t)(sl.h_misc.p[kMiscStatus] & 0xffffffffu);
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, sl.ev0, sl.ev1));
  c->last.tasks = sl.h_misc.p[kMiscCounters];
  c->last.sad_candidates = sl.h_misc.p[kMiscCounters + 1];
  c->last.satd_candidates = sl.h_misc.p[kMiscCounters + 2];
  c->last.sad_samples = sl.h_misc.p[kMiscCounters + 3];
  c->last.satd_samples = sl.h_misc.p[kMiscCounters + 4];
  c->last.kernel_ms = ms;
  if (sl.tuning) {
    auto* T = (Ctx::Tune*)sl.tuning;
    sl.tuning = nullptr;
    if (T->best < 0 && T->tried < kTuneRounds * sl.tune_shapes) {
      // Each shape is timed kTuneRounds times (in turn); its best time counts.
      const int i = T->tried % sl.tune_shapes;
      T->ms[i] = T->tried < sl.tune_shapes ? ms : std::min(T->ms[i], ms);
      if (++T->tried == kTuneRounds * sl.tune_shapes)
        T->best = (int)(std::min_element(T->ms, T->ms + sl.tune_shapes) - T->ms);
    }
  }
  c->last.planes_ms = 0.0f;
  if (c->planes_pending && (wait_planes || cudaEventQuery(c->evp1) == cudaSuccess)) {
    // Device time from the first upload since the previous search to the
    // end of the last one (the uploads' stream precedes this search's).
    cudaEventSynchronize(c->evp1);
    if (cudaEventElapsedTime(&c->last.planes_ms, c->evp0, c->evp1) != cudaSuccess) c->last.planes_ms = 0.0f;
    cudaGetLastError();
    c->planes_pending = false;
  }
  cudaGetLastError();
  if (status) return fail(c, RME_EDEVICE, "device status " + std::to_string(status));
  if (c->last.tasks != (unsigned long long)sl.total)
    return fail(c, RME_EDEVICE, "the launch ran " + std::to_string(c->last.tasks) + " of " + std::to_string(sl.total) +
                                    " tasks");
  if (sl.host_out) {
    for (size_t i = 0; i < sl.host_off.size(); ++i)
      std::memcpy(sl.host_out + sl.host_off[i], sl.h_out.p + sl.dev_off[i], sizeof(rme_result) * sl.host_count[i]);
    sl.host_out = nullptr;
  }
  return 0;
}

// The next slot, free: a launch still in flight there is finished first,
// and an error it reports is kept for its stream's rme_sync.
Slot* take_slot(Ctx* c) {
  Slot& sl = c->slots[c->next_slot];
  c->next_slot = (c->next_slot + 1) % kSlots;
  if (sl.busy) {
    const cudaStream_t st = sl.stream;
    const int rc = finish_launch(c, sl, false);
    if (rc) {
      auto& e = c->async_err[st];
      if (!e.first) e.first = rc;
      if (rc == RME_EDEVICE) e.second |= (uint32_t)(sl.h_misc.p[kMiscStatus] & 0xffffffffu);
    }
  }
  return &sl;
}

// Launch frames[0..n) as one persistent search; results to `out` (device,
// pinned or pageable host memory) at offsets (count-prefix order).
// `bi_src` (HEVC refine_bi): frame 0's per-task target blocks.
// `async`: return once the launch is queued on `s` (out must be device or
// pinned memory); rme_sync finishes it.
int run_launch(Ctx* c, const rme_frame* frames, const rme_params* params, int n, rme_result* out,
               const int64_t* offsets, cudaStream_t s, bool use_graph, const void* bi_src = nullptr,
               bool async = false) {
  if (n < 1 || n > 255) return fail(c, RME_EINVAL, "1..255 frames per launch");
  std::vector<int> ntask(n);
  std::vector<int64_t> toff(n + 1, 0), jobs_off(n + 1, 0);
  for (int i = 0; i < n; ++i) jobs_off[i + 1] = jobs_off[i] + (params[i].predictor_mode == RME_PRED_GIVEN ? frames[i].njobs : 0);
  // `out` may be device memory: the kernels then write it directly.
  cudaPointerAttributes pa{};
  // Pinned host memory takes the results straight from the device buffer.
  const bool known = cudaPointerGetAttributes(&pa, out) == cudaSuccess;
  cudaGetLastError();  // a host pointer unknown to CUDA is not an error here
  const bool dev_out = known && pa.type == cudaMemoryTypeDevice;
  const bool pinned_out = known && pa.type == cudaMemoryTypeHost;
  if (async && !dev_out && !pinned_out)
    return fail(c, RME_EINVAL, "an asynchronous search writes device or pinned host memory only");
  Slot& sl = *take_slot(c);
  // Pass 1: sizes (make_frame with null device pointers validates too).
  CK(sl.h_frames.ensure(n));
  for (int i = 0; i < n; ++i) {
    int rc = make_frame(c, &frames[i], &params[i], &sl.h_frames.p[i], nullptr, nullptr, nullptr, &ntask[i]);
    if (rc) return rc;
    toff[i + 1] = toff[i] + ntask[i];
  }
  const int64_t total = toff[n];
  for (int i = 0; i < n; ++i)
    if (ntask[i] >= (1 << 24)) return fail(c, RME_EINVAL, "more than 2^24 tasks in one frame");
  CK(sl.d_frames.ensure(n));
  if (!dev_out) CK(sl.d_out.ensure(std::max<int64_t>(total, 1)));
  CK(sl.d_pending.ensure(std::max<int64_t>(total, 1)));
  unsigned long long* old_ready = sl.d_ready.p;
  unsigned long long* old_mvf = sl.d_mvf.p;
  CK(sl.d_ready.ensure(2 * std::max<int64_t>(total, 1)));  // the warps' queues, then the CTAs' queues
  CK(sl.d_mvf.ensure(std::max<int64_t>(total, 1)));
  // Fresh slot memory may hold any word, an epoch's among them: zero it
  // (epochs start at 1).
  if (sl.d_ready.p != old_ready || sl.d_mvf.p != old_mvf) sl.epoch = 0;
  CK(sl.d_jobs.ensure(std::max<int64_t>(jobs_off[n], 1)));
  CK(sl.d_misc.ensure(kMiscWords));
  if (!dev_out && !pinned_out) CK(sl.h_out.ensure(std::max<int64_t>(total, 1)));
  CK(sl.h_misc.ensure(kMiscWords));
  if (sl.epoch == 0 || sl.epoch == 0xffffffffu) {
    CK(cudaMemsetAsync(sl.d_ready.p, 0, sl.d_ready.n * sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(sl.d_mvf.p, 0, sl.d_mvf.n * sizeof(unsigned long long), s));
    sl.epoch = 0;
  }
  ++sl.epoch;
  // Pass 2: device pointers; the queue's initial entries (8-bit frames'
  // tasks first, then deeper ones: each part is one kernel launch of its
  // own sample width, with its own part of the slots).
  std::vector<int64_t> sig;
  sig.push_back(n);
  sig.push_back(dev_out + 2 * pinned_out);
  std::vector<unsigned long long> init[kParts], init_big[kParts];
  // A launch of a frame or two is latency-bound: it runs the latency form
  // of the search kernel (same results), where CTAs run the 32x32 and 64x64
  // blocks of HEVC STANDALONE frames together.
  const bool spec = total <= kSpecTasks;
  int64_t part_tasks[kParts] = {0, 0, 0, 0};
  for (int i = 0; i < n; ++i) part_tasks[part_of(sl.h_frames.p[i])] += ntask[i];
  // Each part's launch shape: the tuned one for its class, or the next one
  // to time (a launch of one kind only, so that its time is the part's).
  int nparts_used = 0;
  for (int k = 0; k < kParts; ++k) nparts_used += part_tasks[k] > 0;
  Shape shape[kParts];
  int variant[kParts];
  Ctx::Tune* tuning = nullptr;  // the class this launch times, if any
  int tune_shapes = 0;
  for (int k = 0; k < kParts; ++k) {
    const Shape* shapes = !spec ? kThroughputShapes : part_codec(k) == RME_CODEC_HEVC ? kLatencyHevcShapes : kLatencyShapes;
    const int nsh = kNumShapes[!spec ? 0 : part_codec(k) == RME_CODEC_HEVC ? 1 : 2];
    shape[k] = shapes[0];
    if (part_tasks[k] > 0 && c->tune_on) {
      const int bucket = 63 - __builtin_clzll((unsigned long long)part_tasks[k]);
      Ctx::Tune& T = c->tune[{k * 2 + spec, bucket}];
      if (T.best >= 0) {
        shape[k] = shapes[T.best];
      } else if (nparts_used == 1 && !async) {
        shape[k] = shapes[T.tried % nsh];
        tuning = &T;
        tune_shapes = nsh;
      }
    }
    variant[k] = shape[k].variant;
    if (part_tasks[k] > 0 && !c->bps[k][variant[k]][spec])
      c->bps[k][variant[k]][spec] = search_blocks_per_sm(part_bytes(k), part_codec(k), variant[k], spec);
  }
  // The row form, for a part of the latency form whose frames are all HEVC
  // STANDALONE without AMP when its shape asks for it.
  bool rows[kParts] = {false, false, false, false};
  std::vector<const Deps*> fdeps(n, nullptr);
  for (int k = 0; k < kParts; ++k) rows[k] = spec && part_tasks[k] > 0 && shape[k].rows;
  for (int i = 0; i < n; ++i) {
    const FrameDesc& fd = sl.h_frames.p[i];
    if (params[i].predictor_mode == RME_PRED_STANDALONE) {
      Picture* src;
      picture_of(c, frames[i].src_id, &src);
      int rc = 0;
      fdeps[i] = get_deps(c, src->d, &params[i], frames[i].nref, &rc);
      if (!fdeps[i]) return rc;
    }
    if (fd.codec != RME_CODEC_HEVC || params[i].predictor_mode != RME_PRED_STANDALONE || fd.amp != 0)
      rows[part_of(fd)] = false;
  }
  int64_t rows_small[kParts] = {0, 0, 0, 0}, rows_large[kParts] = {0, 0, 0, 0};
  std::vector<std::pair<const int32_t*, int>> pend_copies;  // (template, frame)
  for (int i = 0; i < n; ++i) {
    FrameDesc& fd = sl.h_frames.p[i];
    const int part = part_of(fd);
    fd.out = dev_out ? out + (offsets ? offsets[i] : toff[i]) : sl.d_out.p + toff[i];
    fd.pending = sl.d_pending.p + toff[i];
    const unsigned long long tag = ((unsigned long long)sl.epoch << 32) | ((unsigned long long)i << 24);
    if (params[i].predictor_mode == RME_PRED_GIVEN) {
      fd.jobs = sl.d_jobs.p + jobs_off[i];
      if (i == 0) fd.bi_src = bi_src;
      if (frames[i].njobs > 0)
        CK(cudaMemcpyAsync(sl.d_jobs.p + jobs_off[i], frames[i].jobs, sizeof(rme_job) * frames[i].njobs,
                           cudaMemcpyHostToDevice, s));
      for (int t = 0; t < ntask[i]; ++t) init[part].push_back(tag | (uint32_t)t);
      sig.push_back(-1);
      sig.push_back(frames[i].njobs);
      sig.push_back(fd.bd);
    } else if (rows[part]) {
      // Every row of the frame is pushed now (interleaved with the other
      // frames' rows below); a search of this buffer tags its words anew.
      const Deps* dp = fdeps[i];
      fd.mvf = sl.d_mvf.p + toff[i];
      fd.tag = sl.epoch;
      fd.nrows = (int32_t)(dp->rows.size() + dp->rows_big.size());
      rows_small[part] += (int64_t)dp->rows.size();
      rows_large[part] += (int64_t)dp->rows_big.size();
      sig.push_back(fd.bd);
      sig.push_back(fd.codec);
      sig.push_back(fd.width);
      sig.push_back(fd.height);
      sig.push_back(fd.nref);
      sig.push_back(params[i].hevc_pu_mask);
    } else {
      const Deps* dp = fdeps[i];
      pend_copies.emplace_back(dp->pending, i);
      const bool groups = spec && fd.codec == RME_CODEC_HEVC && shape[part].groups > 0;
      for (uint32_t t : dp->ready)
        (groups && (int)(t / fd.nref) < fd.big_end ? init_big : init)[part].push_back(tag | t);
      sig.push_back(fd.bd);
      sig.push_back(fd.codec);
      sig.push_back(fd.width);
      sig.push_back(fd.height);
      sig.push_back(fd.nref);
      sig.push_back(params[i].hevc_pu_mask);
    }
  }
  // Frames' first tasks interleaved, so every frame starts at once.
  for (int k = 0; k < kParts; ++k)
    for (auto* v : {&init[k], &init_big[k]})
      std::stable_sort(v->begin(), v->end(), [](unsigned long long a, unsigned long long b) {
        return (a & 0xffffffu) < (b & 0xffffffu);
      });
  // Row-form parts: the frames' rows interleaved row for row (each frame's
  // own order kept).
  for (int k = 0; k < kParts; ++k) {
    if (!rows[k]) continue;
    for (int big = 0; big < 2; ++big) {
      auto list = [&](int i) -> const std::vector<uint32_t>& { return big ? fdeps[i]->rows_big : fdeps[i]->rows; };
      size_t most = 0;
      for (int i = 0; i < n; ++i)
        if (part_of(sl.h_frames.p[i]) == k) most = std::max(most, list(i).size());
      for (size_t j = 0; j < most; ++j)
        for (int i = 0; i < n; ++i) {
          if (part_of(sl.h_frames.p[i]) != k) continue;
          const std::vector<uint32_t>& v = list(i);
          if (j < v.size())
            (big ? init_big : init)[k].push_back(((unsigned long long)sl.epoch << 32) |
                                                 ((unsigned long long)i << 24) | v[j]);
        }
    }
  }
  // h_init: [the launch header (kMiscWords) | entries | the CTAs' entries]
  size_t ninit = 0, init_off[kParts], init_big_off[kParts];
  for (int k = 0; k < kParts; ++k) {
    init_off[k] = ninit;
    ninit += init[k].size();
  }
  for (int k = 0; k < kParts; ++k) {
    init_big_off[k] = ninit;
    ninit += init_big[k].size();
  }
  CK(sl.h_init.ensure(kMiscWords + ninit));
  unsigned long long* hi = sl.h_init.p;
  std::memset(hi, 0, kMiscWords * sizeof(unsigned long long));
  hi[kMiscEpoch] = sl.epoch;
  LaunchDesc Ls[kParts] = {};
  int64_t slot0 = 0, slot_off[kParts];
  for (int k = 0; k < kParts; ++k) {
    hi[2 * k + 1] = init[k].size();
    hi[kMiscBig + 2 * k + 1] = init_big[k].size();
    std::memcpy(hi + kMiscWords + init_off[k], init[k].data(), init[k].size() * sizeof(unsigned long long));
    std::memcpy(hi + kMiscWords + init_big_off[k], init_big[k].data(), init_big[k].size() * sizeof(unsigned long long));
    slot_off[k] = slot0;
    LaunchDesc& L = Ls[k];
    L.frames = sl.d_frames.p;
    L.ready = sl.d_ready.p + slot0;
    L.total = part_tasks[k];
    L.head = sl.d_misc.p + 2 * k;
    L.tail = sl.d_misc.p + 2 * k + 1;
    L.counters = sl.d_misc.p + kMiscCounters;
    L.status = reinterpret_cast<uint32_t*>(sl.d_misc.p + kMiscStatus);
    L.epoch = reinterpret_cast<const uint32_t*>(sl.d_misc.p + kMiscEpoch);
    L.done = sl.d_misc.p + kMiscDone + k;
    L.ready_big = sl.d_ready.p + total + slot0;
    L.head_big = sl.d_misc.p + kMiscBig + 2 * k;
    L.tail_big = sl.d_misc.p + kMiscBig + 2 * k + 1;
    L.group_ctas = 0;
    if (rows[k]) {
      L.rows = 1;
      L.total = rows_small[k];
      L.total_big = rows_large[k];
      L.done = nullptr;
    }
    slot0 += part_tasks[k];
  }
  for (int k = 0; k < kParts; ++k) {
    sig.push_back(variant[k]);
    sig.push_back(shape[k].patch);
    sig.push_back(rows[k]);
    Ls[k].patch8 = shape[k].patch;
  }
  int nparts = 0, order[kParts];
  for (int k = 0; k < kParts; ++k)
    if (part_tasks[k] > 0) order[nparts++] = k;
  for (int j = 1; j < nparts; ++j) {
    if (!c->aux[j]) CK(cudaStreamCreateWithFlags(&c->aux[j], cudaStreamNonBlocking));
    if (!c->ev_join[j]) CK(cudaEventCreateWithFlags(&c->ev_join[j], cudaEventDisableTiming));
  }
  if (nparts > 1 && !c->ev_fork) CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  sig.push_back(nparts);
  // Grids: in the latency form a part with large HEVC blocks gives them up
  // to half the SMs' worth of CTAs (one block at a time each) and the rest to
  // the warps; all CTAs fit on the GPU at once, so neither kind waits for
  // the other to be scheduled.
  int grid[kParts] = {0, 0, 0, 0};
  for (int k = 0; k < kParts; ++k) {
    if (part_tasks[k] == 0) continue;
    const int cap = c->nsm * c->bps[k][variant[k]][spec];
    int64_t big = 0;
    if (spec && part_codec(k) == RME_CODEC_HEVC)
      for (int i = 0; i < n; ++i)
        if (part_of(sl.h_frames.p[i]) == k && params[i].predictor_mode == RME_PRED_STANDALONE)
          big += (int64_t)sl.h_frames.p[i].big_end * sl.h_frames.p[i].nref;
    const int share = shape[k].groups == 3 ? cap / 2
                      : shape[k].groups == 2 ? c->nsm / 2
                      : shape[k].groups == 1 ? c->nsm / 4
                                             : 0;
    int g = big > 0 && share > 0 ? (int)std::min<int64_t>({(int64_t)share, big, (int64_t)cap - 1}) : 0;
    int64_t small = part_tasks[k] - big;
    if (rows[k]) {
      // A CTA per row of large blocks (at least one when there are any), a
      // warp per row of small ones.
      g = rows_large[k] > 0
              ? (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)std::max(share, 1), rows_large[k], (int64_t)cap - 1}))
              : 0;
      small = rows_small[k];
    }
    const int solo = (int)std::max<int64_t>(1, std::min<int64_t>(cap - g, (small + kWarpsPerBlock - 1) / kWarpsPerBlock));
    Ls[k].group_ctas = g;
    grid[k] = g + solo;
    sig.push_back(g);
  }
  auto enqueue = [&](bool capturing) -> cudaError_t {
    const unsigned rec = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    cudaError_t e = cudaMemcpyAsync(sl.d_frames.p, sl.h_frames.p, sizeof(FrameDesc) * n, cudaMemcpyHostToDevice, s);
    for (auto& pc : pend_copies)
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(sl.d_pending.p + toff[pc.second], pc.first, sizeof(int32_t) * ntask[pc.second],
                            cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sl.d_misc.p, hi, kMiscWords * sizeof(unsigned long long), cudaMemcpyHostToDevice, s);
    for (int k = 0; k < kParts; ++k) {
      if (e == cudaSuccess && !init[k].empty())
        e = cudaMemcpyAsync(sl.d_ready.p + slot_off[k], hi + kMiscWords + init_off[k],
                            init[k].size() * sizeof(unsigned long long), cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess && !init_big[k].empty())
        e = cudaMemcpyAsync(sl.d_ready.p + total + slot_off[k], hi + kMiscWords + init_big_off[k],
                            init_big[k].size() * sizeof(unsigned long long), cudaMemcpyHostToDevice, s);
    }
    // Under capture the records are external ones: they become event-record
    // nodes, so the kernels' device time is measured on every replay.
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(sl.ev0, s, rec);
    // Parts after the first run concurrently on the auxiliary streams
    // (parallel branches of a captured graph).
    if (e == cudaSuccess && nparts > 1) e = cudaEventRecord(c->ev_fork, s);
    for (int j = 0; j < nparts && e == cudaSuccess; ++j) {
      const int k = order[j];
      cudaStream_t sk = j == 0 ? s : c->aux[j];
      if (j > 0) e = cudaStreamWaitEvent(sk, c->ev_fork, 0);
      if (e == cudaSuccess)
        e = launch_search(Ls[k], part_bytes(k), part_codec(k), variant[k], grid[k], sk, spec);
      if (e == cudaSuccess && j > 0) e = cudaEventRecord(c->ev_join[j], sk);
    }
    for (int j = 1; j < nparts && e == cudaSuccess; ++j) e = cudaStreamWaitEvent(s, c->ev_join[j], 0);
    if (e == cudaSuccess) e = cudaEventRecordWithFlags(sl.ev1, s, rec);
    if (e == cudaSuccess && !dev_out && !pinned_out)
      e = cudaMemcpyAsync(sl.h_out.p, sl.d_out.p, sizeof(rme_result) * total, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sl.h_misc.p, sl.d_misc.p, kMiscWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    return e;
  };
  bool has_given = false;
  for (int i = 0; i < n; ++i) has_given |= params[i].predictor_mode == RME_PRED_GIVEN;
  if (use_graph && !has_given) {
    std::vector<int64_t> gsig = sig;
    gsig.push_back(total);
    for (int k = 0; k < kParts; ++k) gsig.push_back((int64_t)init[k].size());
    gsig.push_back((int64_t)(uintptr_t)s);
    gsig.push_back((int64_t)(&sl - c->slots));
    gsig.push_back((int64_t)g_buffer_generation);
    Graph& g = c->graphs[gsig];
    // A shape is captured when it comes a second time (a one-off batch,
    // common in serving, is not worth a capture).
    if (!g.exec && ++g.seen < 2) {
      CK(enqueue(false));
    } else if (!g.exec) {
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = enqueue(true);
      cudaError_t e2 = cudaStreamEndCapture(s, &graph);
      if (e != cudaSuccess) return cuda_fail(c, e, "graph capture");
      if (e2 != cudaSuccess) return cuda_fail(c, e2, "graph capture end");
      e = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        g.exec = nullptr;
        return cuda_fail(c, e, "graph instantiate");
      }
    }
    if (g.exec) CK(cudaGraphLaunch(g.exec, s));
  } else {
    CK(enqueue(false));
  }
  if (pinned_out) {
    // One copy per run of frames whose results are contiguous in `out`.
    for (int i = 0; i < n;) {
      int j = i + 1;
      while (j < n && (!offsets || offsets[j] == offsets[i] + (toff[j] - toff[i]))) ++j;
      const int64_t off = offsets ? offsets[i] : toff[i];
      if (toff[j] > toff[i])
        CK(cudaMemcpyAsync(out + off, sl.d_out.p + toff[i], sizeof(rme_result) * (toff[j] - toff[i]),
                           cudaMemcpyDeviceToHost, s));
      i = j;
    }
  }
  CK(cudaEventRecord(sl.done, s));
  sl.busy = true;
  sl.stream = s;
  sl.total = total;
  sl.tuning = tuning;
  sl.tune_shapes = tune_shapes;
  if (!dev_out && !pinned_out) {
    sl.host_out = out;
    sl.host_off.resize(n);
    sl.host_count.resize(n);
    sl.dev_off.resize(n);
    for (int i = 0; i < n; ++i) {
      sl.host_off[i] = offsets ? offsets[i] : toff[i];
      sl.host_count[i] = ntask[i];
      sl.dev_off[i] = toff[i];
    }
  }
  if (async) return 0;
  return finish_launch(c, sl);
}

}  // namespace

namespace rme {
// A STANDALONE frame for the resident engine: its descriptor over the
// context's pictures (launch buffers left null), its task count, its
// dependency template and its root tasks (device memory, held by the
// context).
int ctx_standalone_frame(void* ctx, const rme_frame* f, const rme_params* p, FrameDesc* fd, int* ntasks,
                         const int32_t** pending_tmpl, const uint32_t** roots, int* nroots) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !f || !p || !fd || !ntasks) return RME_EINVAL;
  if (p->predictor_mode != RME_PRED_STANDALONE) return fail(c, RME_EINVAL, "the engine searches STANDALONE frames");
  int rc = make_frame(c, f, p, fd, nullptr, nullptr, nullptr, ntasks);
  if (rc) return rc;
  if (*ntasks >= (1 << 24)) return fail(c, RME_EINVAL, "more than 2^24 tasks in one frame");
  Picture* src;
  if ((rc = picture_of(c, f->src_id, &src))) return rc;
  const Deps* dp = get_deps(c, src->d, p, f->nref, &rc);
  if (!dp) return rc;
  *pending_tmpl = dp->pending;
  *roots = dp->d_ready;
  *nroots = (int)dp->ready.size();
  return 0;
}

bool ctx_frame_rows(void* ctx, const rme_frame* f, const rme_params* p, const uint32_t** rows, int* nrows,
                    const uint32_t** rows_big, int* nrows_big) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !f || !p || p->predictor_mode != RME_PRED_STANDALONE || p->hevc_amp != 0) return false;
  auto it = c->pics.find(f->src_id);
  if (it == c->pics.end() || it->second->d.codec != RME_CODEC_HEVC) return false;
  int rc = 0;
  const Deps* dp = get_deps(c, it->second->d, p, f->nref, &rc);
  if (!dp || !dp->d_rows) return false;
  *rows = dp->d_rows;
  *nrows = (int)dp->rows.size();
  *rows_big = dp->d_rows + dp->rows.size();
  *nrows_big = (int)dp->rows_big.size();
  return true;
}
}  // namespace rme

extern "C" {

void rme_params_default(rme_params* p, int32_t codec, int32_t qp) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->codec = codec;
  p->qp = qp;
  p->predictor_mode = RME_PRED_STANDALONE;
  p->h264_range = 16;
  p->h264_hpel_iters = 2;
  p->h264_qpel_iters = 2;
  p->h264_refine_ratio = 1.5f;
  p->h264_vertical_range = 0x7ffffffe;
  p->h264_pad = kH264Pad;
  p->hevc_search_range = 48;
  p->hevc_search_rings = 0;
  p->hevc_quarter_cross = 0;
  p->hevc_lambda_scale = 0.85f;
  p->hevc_pad = kHevcPad;
  p->hevc_pu_mask = 0xF;
  p->hevc_amp = 0;
}

int rme_ctx_create(void** out, int32_t device) {
  if (!out) return RME_EINVAL;
  *out = nullptr;
  auto c = std::make_unique<Ctx>();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return RME_ECUDA;
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return RME_ECUDA;
  c->nsm = nsm;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return RME_ECUDA;
  // RME_TUNE=0 keeps every launch on the default occupancy variant.
  if (const char* t = std::getenv("RME_TUNE")) c->tune_on = t[0] != '0';
  if (cudaEventCreate(&c->evp0) != cudaSuccess || cudaEventCreate(&c->evp1) != cudaSuccess) return RME_ECUDA;
  for (Slot& sl : c->slots)
    if (cudaEventCreate(&sl.ev0) != cudaSuccess || cudaEventCreate(&sl.ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess)
      return RME_ECUDA;
  *out = c.release();
  return 0;
}

void rme_ctx_destroy(void* ctx) {
  if (!ctx) return;
  Ctx* c = (Ctx*)ctx;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  delete c;
}

const char* rme_last_error(void* ctx) { return ctx ? ((Ctx*)ctx)->err.c_str() : "null context"; }

namespace {
// A picture's device layout (no memory yet): H.264 planes at the coded
// (macroblock) size, HEVC at the picture's; rows of 128-byte multiples, the
// visible origin 16-byte aligned (pad * bytes is a multiple of 16 for both
// pads); a reference holds its search planes after plane 0.
std::unique_ptr<Picture> picture_geometry(const rme_picture_desc* d, bool as_ref) {
  auto pic = std::make_unique<Picture>();
  pic->d = *d;
  const bool h264 = d->codec == RME_CODEC_H264;
  pic->cw = h264 ? (d->width + 15) / 16 * 16 : d->width;
  pic->ch = h264 ? (d->height + 15) / 16 * 16 : d->height;
  pic->pad = h264 ? kH264Pad : kHevcPad;
  pic->is_ref = as_ref;
  pic->nplanes = as_ref ? (h264 ? 4 : 16) : 1;
  const int bps = d->bit_depth == 8 ? 1 : 2;
  const int stride_bytes = ((pic->cw + 2 * pic->pad) * bps + 127) / 128 * 128;
  const int stride = stride_bytes / bps, rows = pic->ch + 2 * pic->pad;
  pic->planes.stride = stride;
  pic->planes.plane_elems = (int64_t)stride * rows;
  pic->planes.origin = pic->pad * stride + pic->pad;
  pic->bytes = (size_t)pic->planes.plane_elems * bps * pic->nplanes + 256;
  return pic;
}

// The device buffer of picture `id`'s new contents: the old entry's when
// the geometry matches (a stream's picture slots are refilled every frame;
// work already queued on the old contents is ordered before the refill by
// the stream), else a fresh one. The old entry leaves the table here, so a
// failure after this leaves the id unknown instead of naming a picture
// without a buffer.
cudaError_t take_buffer(Ctx* c, int32_t id, Picture* pic, cudaStream_t s) {
  auto old = c->pics.find(id);
  if (old != c->pics.end()) {
    if (old->second->bytes == pic->bytes && old->second->planes.stride == pic->planes.stride) {
      pic->buf = old->second->buf;
      old->second->buf = nullptr;
    } else {
      cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return e;
    }
    c->pics.erase(old);
  }
  if (!pic->buf) {
    cudaError_t e = cudaMalloc(&pic->buf, pic->bytes);
    if (e != cudaSuccess) return e;
  }
  pic->planes.base = pic->buf;
  return cudaSuccess;
}
}  // namespace

int rme_picture_upload(void* ctx, int32_t pic_id, const rme_picture_desc* d, const void* luma, int32_t as_ref,
                       void* stream) {
  return rme::ctx_picture_upload(ctx, pic_id, d, luma, as_ref, as_ref != 0, stream);
}

}  // extern "C"

namespace rme {
int ctx_picture_upload(void* ctx, int32_t pic_id, const rme_picture_desc* d, const void* luma, int32_t as_ref,
                       bool build_planes, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (!valid_desc(d) || !luma || pic_id < 0) return fail(c, RME_EINVAL, "bad picture description");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  auto pic = picture_geometry(d, as_ref != 0);
  const bool h264 = d->codec == RME_CODEC_H264;
  const int bps = d->bit_depth == 8 ? 1 : 2, stride = pic->planes.stride;
  CK(take_buffer(c, pic_id, pic.get(), s));
  // The visible picture straight into plane 0, then its border in place:
  // nothing is staged, so nothing waits (a pageable source is consumed
  // before the copy call returns; a pinned one is read on the stream).
  uint8_t* origin = (uint8_t*)pic->buf + (size_t)pic->planes.origin * bps;
  if (!c->planes_pending) CK(cudaEventRecord(c->evp0, s));
  CK(cudaMemcpy2DAsync(origin, (size_t)stride * bps, luma, (size_t)d->stride * bps, (size_t)d->width * bps, d->height,
                       cudaMemcpyHostToDevice, s));
  CK(launch_pad_plane(origin, d->bit_depth, d->width, d->height, stride, pic->planes, pic->cw, pic->ch, pic->pad, s));
  if (as_ref && build_planes) {
    if (h264) CK(launch_h264_hpel(pic->planes, d->bit_depth, pic->cw, pic->ch, pic->pad, s));
    else CK(launch_hevc_phases(pic->planes, d->bit_depth, pic->cw, pic->ch, pic->pad, s));
  }
  CK(cudaEventRecord(c->evp1, s));
  c->planes_pending = true;
  c->pics[pic_id] = std::move(pic);
  return 0;
}
}  // namespace rme

extern "C" {

int rme_picture_upload_chroma(void* ctx, int32_t pic_id, const void* cb, const void* cr, int32_t cstride,
                              void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  Picture* p;
  int rc = picture_of(c, pic_id, &p);
  if (rc) return rc;
  if (!cb || !cr || cstride < p->d.width / 2) return fail(c, RME_EINVAL, "bad chroma planes");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  int bps = p->d.bit_depth == 8 ? 1 : 2, w = p->d.width / 2, h = p->d.height / 2;
  if (p->chroma) cudaFree(p->chroma);
  p->chroma = nullptr;
  p->chroma_bytes = (size_t)w * h * bps * 2;
  CK(cudaMalloc(&p->chroma, p->chroma_bytes + 64));
  CK(cudaMemcpy2DAsync(p->chroma, (size_t)w * bps, cb, (size_t)cstride * bps, (size_t)w * bps, h,
                       cudaMemcpyHostToDevice, s));
  CK(cudaMemcpy2DAsync((uint8_t*)p->chroma + (size_t)w * h * bps, (size_t)w * bps, cr, (size_t)cstride * bps,
                       (size_t)w * bps, h, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_picture_release(void* ctx, int32_t pic_id) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  auto it = c->pics.find(pic_id);
  if (it == c->pics.end()) return fail(c, RME_ENOTFOUND, "picture not uploaded");
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->pics.erase(it);
  return 0;
}

int rme_picture_build_planes(void* ctx, int32_t pic_id, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  Picture* p;
  int rc = picture_of(c, pic_id, &p);
  if (rc) return rc;
  if (!p->is_ref) return fail(c, RME_EINVAL, "picture was uploaded without as_ref");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  if (p->d.codec == RME_CODEC_H264) CK(launch_h264_hpel(p->planes, p->d.bit_depth, p->cw, p->ch, p->pad, s));
  else CK(launch_hevc_phases(p->planes, p->d.bit_depth, p->cw, p->ch, p->pad, s));
  return 0;
}

// ---- weighted prediction (h264_me.rs / h265_me.rs weighted_search_plane,
// distortion.rs wp_moments / weighted_sad) ------------------------------------

int rme_picture_weighted(void* ctx, int32_t ref_id, int32_t dst_id, int32_t log_wd, int32_t weight, int32_t offset,
                         void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  Picture* p;
  int rc = picture_of(c, ref_id, &p);
  if (rc) return rc;
  if (!p->is_ref) return fail(c, RME_EINVAL, "picture was uploaded without as_ref");
  if (dst_id < 0 || dst_id == ref_id) return fail(c, RME_EINVAL, "the weighted plane needs an id of its own");
  const bool h264 = p->d.codec == RME_CODEC_H264;
  if (log_wd < (h264 ? 0 : 1) || log_wd > 14 || weight < -128 || weight > 255 || offset < -(1 << p->d.bit_depth) ||
      offset > (1 << p->d.bit_depth))
    return fail(c, RME_EINVAL, "weighting out of range");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  auto pic = picture_geometry(&p->d, true);
  CK(take_buffer(c, dst_id, pic.get(), s));
  const int bps = p->d.bit_depth == 8 ? 1 : 2;
  CK(launch_weighted_plane(p->buf, pic->buf, pic->planes.plane_elems * bps, p->d.codec, p->d.bit_depth, log_wd, weight,
                           offset, s));
  if (h264) CK(launch_h264_hpel(pic->planes, p->d.bit_depth, pic->cw, pic->ch, pic->pad, s));
  else CK(launch_hevc_phases(pic->planes, p->d.bit_depth, pic->cw, pic->ch, pic->pad, s));
  c->pics[dst_id] = std::move(pic);
  return 0;
}

namespace {
int picture_pair(Ctx* c, int32_t cur_id, int32_t ref_id, Picture** pc, Picture** pr) {
  int rc = picture_of(c, cur_id, pc);
  if (!rc) rc = picture_of(c, ref_id, pr);
  if (rc) return rc;
  const rme_picture_desc &a = (*pc)->d, &b = (*pr)->d;
  if (a.codec != b.codec || a.bit_depth != b.bit_depth || a.width != b.width || a.height != b.height ||
      (*pc)->planes.stride != (*pr)->planes.stride)
    return fail(c, RME_EINVAL, "the pictures' formats differ");
  return 0;
}
}  // namespace

int rme_wp_moments(void* ctx, int32_t cur_id, int32_t ref_id, uint64_t* out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !out) return c ? fail(c, RME_EINVAL, "null argument") : RME_EINVAL;
  Picture *pc, *pr;
  int rc = picture_pair(c, cur_id, ref_id, &pc, &pr);
  if (rc) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  CK(c->d_wp.ensure(8));
  CK(cudaMemsetAsync(c->d_wp.p, 0, 5 * sizeof(unsigned long long), s));
  const int bps = pc->d.bit_depth == 8 ? 1 : 2;
  CK(launch_wp_moments((const uint8_t*)pc->buf + (size_t)pc->planes.origin * bps,
                       (const uint8_t*)pr->buf + (size_t)pr->planes.origin * bps, pc->planes.stride, pc->d.bit_depth,
                       pc->d.width, pc->d.height, c->d_wp.p, s));
  CK(cudaMemcpyAsync(out, c->d_wp.p, 5 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_weighted_sad(void* ctx, int32_t cur_id, int32_t ref_id, int32_t weight, int32_t shift, int32_t offset,
                     uint64_t* out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !out) return c ? fail(c, RME_EINVAL, "null argument") : RME_EINVAL;
  if (shift < 0 || shift > 14 || weight < -128 || weight > 255) return fail(c, RME_EINVAL, "weighting out of range");
  Picture *pc, *pr;
  int rc = picture_pair(c, cur_id, ref_id, &pc, &pr);
  if (rc) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  CK(c->d_wp.ensure(8));
  CK(cudaMemsetAsync(c->d_wp.p + 5, 0, sizeof(unsigned long long), s));
  const int bps = pc->d.bit_depth == 8 ? 1 : 2;
  CK(launch_weighted_sad((const uint8_t*)pc->buf + (size_t)pc->planes.origin * bps,
                         (const uint8_t*)pr->buf + (size_t)pr->planes.origin * bps, pc->planes.stride,
                         pc->d.bit_depth, pc->d.width, pc->d.height, weight, shift, offset, c->d_wp.p + 5, s));
  CK(cudaMemcpyAsync(out, c->d_wp.p + 5, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_picture_download_plane(void* ctx, int32_t pic_id, int32_t plane, void* out, int32_t* rows, int32_t* cols) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  Picture* p;
  int rc = picture_of(c, pic_id, &p);
  if (rc) return rc;
  if (plane < 0 || plane >= p->nplanes) return fail(c, RME_EINVAL, "plane index out of range");
  int R = p->ch + 2 * p->pad, C = p->cw + 2 * p->pad, bps = p->d.bit_depth == 8 ? 1 : 2;
  if (rows) *rows = R;
  if (cols) *cols = C;
  if (!out) return 0;
  const uint8_t* src = (const uint8_t*)p->buf + (size_t)plane * p->planes.plane_elems * bps;
  CK(cudaMemcpy2D(out, (size_t)C * bps, src, (size_t)p->planes.stride * bps, (size_t)C * bps, R,
                  cudaMemcpyDeviceToHost));
  return 0;
}

int rme_memory_used(void* ctx, uint64_t* bytes) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !bytes) return RME_EINVAL;
  uint64_t b = 0;
  for (auto& kv : c->pics) b += kv.second->bytes + kv.second->chroma_bytes;
  *bytes = b;
  return 0;
}

int rme_standalone_blocks(const rme_picture_desc* d, const rme_params* p, int32_t* blocks, int32_t* count) {
  if (!valid_desc(d) || !p || !count) return RME_EINVAL;
  *count = count_blocks(d, p, blocks);
  return 0;
}

int rme_frame_result_count(void* ctx, const rme_frame* f, const rme_params* p, int32_t* count) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !f || !p || !count) return RME_EINVAL;
  if (p->predictor_mode == RME_PRED_GIVEN) {
    *count = f->njobs;
    return 0;
  }
  Picture* src;
  int rc = picture_of(c, f->src_id, &src);
  if (rc) return rc;
  int nb = count_blocks(&src->d, p, nullptr);
  *count = src->d.codec == RME_CODEC_H264 ? nb : nb * f->nref;
  return 0;
}

int rme_frame_search(void* ctx, const rme_frame* f, const rme_params* p, rme_result* out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !f || !p || !out) return c ? fail(c, RME_EINVAL, "null argument") : RME_EINVAL;
  CK(cudaSetDevice(c->device));
  return run_launch(c, f, p, 1, out, nullptr, stream ? (cudaStream_t)stream : c->stream, false);
}

int rme_batch_search(void* ctx, const rme_frame* frames, const rme_params* params, int32_t nframes, rme_result* out,
                     const int64_t* offsets, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !frames || !params || !out || nframes < 1) return c ? fail(c, RME_EINVAL, "null argument") : RME_EINVAL;
  CK(cudaSetDevice(c->device));
  return run_launch(c, frames, params, nframes, out, offsets, stream ? (cudaStream_t)stream : c->stream, true);
}

int rme_frame_search_async(void* ctx, const rme_frame* f, const rme_params* p, rme_result* out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !f || !p || !out) return c ? fail(c, RME_EINVAL, "null argument") : RME_EINVAL;
  CK(cudaSetDevice(c->device));
  return run_launch(c, f, p, 1, out, nullptr, stream ? (cudaStream_t)stream : c->stream, false, nullptr, true);
}

int rme_batch_search_async(void* ctx, const rme_frame* frames, const rme_params* params, int32_t nframes,
                           rme_result* out, const int64_t* offsets, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !frames || !params || !out || nframes < 1) return c ? fail(c, RME_EINVAL, "null argument") : RME_EINVAL;
  CK(cudaSetDevice(c->device));
  return run_launch(c, frames, params, nframes, out, offsets, stream ? (cudaStream_t)stream : c->stream, false,
                    nullptr, true);
}

int rme_sync(void* ctx, void* stream, uint32_t* device_status) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  CK(cudaSetDevice(c->device));
  const cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  int rc = 0;
  uint32_t st = 0;
  auto it = c->async_err.find(s);
  if (it != c->async_err.end()) {
    rc = it->second.first;
    st = it->second.second;
    c->async_err.erase(it);
  }
  // Oldest first: the slot after the last one taken, round the ring.
  for (int k = 0; k < kSlots; ++k) {
    Slot& sl = c->slots[(c->next_slot + k) % kSlots];
    if (!sl.busy || sl.stream != s) continue;
    const int r = finish_launch(c, sl, false);
    if (r == RME_EDEVICE) st |= (uint32_t)(sl.h_misc.p[kMiscStatus] & 0xffffffffu);
    if (r && !rc) rc = r;
  }
  if (device_status) *device_status = st;
  return rc;
}

int rme_hevc_decide(const rme_picture_desc* d, const rme_params* p, int32_t nref, const rme_result* res,
                    int32_t* best, uint8_t* part) {
  if (!valid_desc(d) || !p || !res || nref < 1 || nref > RME_MAX_REFS || d->codec != RME_CODEC_HEVC)
    return RME_EINVAL;
  int W = d->width, H = d->height;
  float lam = hevc_lambda(p->qp, d->bit_depth, p->hevc_lambda_scale);
  int sizes[4], nl = level_sizes(p, sizes);
  int base[5] = {0}, nbx[4], nby[4];
  for (int l = 0; l < nl; ++l) {
    nbx[l] = W / sizes[l];
    nby[l] = H / sizes[l];
    base[l + 1] = base[l] + nbx[l] * nby[l];
  }
  const int nb_all = count_blocks(d, p, nullptr);  // AMP units included
  std::vector<uint64_t> cost(nb_all);
  for (int b = 0; b < nb_all; ++b) {
    int br = 0;
    uint64_t bc = UINT64_MAX;
    for (int r = 0; r < nref; ++r) {
      uint64_t cc = (uint64_t)res[(size_t)b * nref + r].cost + (uint32_t)(lam * (float)hevc_ref_idx_bits(r, nref));
      if (cc < bc) {
        bc = cc;
        br = r;
      }
    }
    cost[b] = bc;
    if (best) best[b] = br;
  }
  if (!part) return 0;
  int cw = W / 8, ch = H / 8;
  std::memset(part, 0, (size_t)cw * ch);
  // Iterative bottom-up: the least cost of every node of every level.
  std::vector<std::vector<uint64_t>> node(nl);
  std::vector<std::vector<uint8_t>> split(nl);
  for (int l = nl - 1; l >= 0; --l) {
    int N = sizes[l], gx = (W + N - 1) / N, gy = (H + N - 1) / N;
    node[l].assign((size_t)gx * gy, UINT64_MAX);
    split[l].assign((size_t)gx * gy, 0);
    for (int y = 0; y < gy; ++y)
      for (int x = 0; x < gx; ++x) {
        int px = x * N, py = y * N;
        bool exists = px + N <= W && py + N <= H;
        uint64_t own = exists ? cost[base[l] + y * nbx[l] + x] : UINT64_MAX;
        uint64_t sp = UINT64_MAX;
        if (l + 1 < nl) {
          int M = sizes[l + 1], cgx = (W + M - 1) / M;
          sp = 0;
          for (int yy = py; yy < py + N && sp != UINT64_MAX; yy += M)
            for (int xx = px; xx < px + N; xx += M) {
              if (xx >= W || yy >= H) continue;
              uint64_t cc = node[l + 1][(size_t)(yy / M) * cgx + xx / M];
              if (cc == UINT64_MAX) {
                sp = UINT64_MAX;
                break;
              }
              sp += cc;
            }
        }
        bool s = sp < own;
        split[l][(size_t)y * gx + x] = s;
        node[l][(size_t)y * gx + x] = s ? sp : own;
      }
  }
  // Top-down marking of the chosen sizes.
  std::vector<std::tuple<int, int, int>> st;
  int N0 = sizes[0];
  for (int y = 0; y < H; y += N0)
    for (int x = 0; x < W; x += N0) st.emplace_back(0, x, y);
  while (!st.empty()) {
    auto [l, px, py] = st.back();
    st.pop_back();
    int N = sizes[l], gx = (W + N - 1) / N;
    size_t idx = (size_t)(py / N) * gx + px / N;
    if (split[l][idx]) {
      int M = sizes[l + 1];
      for (int yy = py; yy < py + N; yy += M)
        for (int xx = px; xx < px + N; xx += M)
          if (xx < W && yy < H) st.emplace_back(l + 1, xx, yy);
    } else if (px + N <= W && py + N <= H && node[l][idx] != UINT64_MAX) {
      int lg = 31 - __builtin_clz((unsigned)N);
      for (int yy = py / 8; yy < (py + N) / 8 && yy < ch; ++yy)
        for (int xx = px / 8; xx < (px + N) / 8 && xx < cw; ++xx) part[yy * cw + xx] = (uint8_t)lg;
    }
  }
  return 0;
}

int rme_last_stats(void* ctx, rme_stats* s) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !s) return RME_EINVAL;
  *s = c->last;
  return 0;
}

// ---- B pictures: bi-prediction (h265_me.rs satd_bi_at, refine_bi) -------------

namespace {
// The frame's source and references, checked as make_frame checks them, and
// the jobs copied to the device.
int bi_setup(Ctx* c, const rme_frame* f, const rme_params* p, const rme_bi_job* jobs, int32_t n, bool refine,
             cudaStream_t s, BiDesc* B) {
  if (!f || !p || n < 0 || (n > 0 && !jobs)) return fail(c, RME_EINVAL, "null argument");
  Picture* src;
  int rc = picture_of(c, f->src_id, &src);
  if (rc) return rc;
  if (src->d.codec != RME_CODEC_HEVC) return fail(c, RME_EINVAL, "bi-prediction jobs are HEVC's");
  if (f->nref < 1 || f->nref > RME_MAX_REFS) return fail(c, RME_EINVAL, "nref must be 1..4");
  if ((rc = check_params(c, p, src->d))) return rc;
  std::memset(B, 0, sizeof(*B));
  B->src = src->planes;
  for (int r = 0; r < f->nref; ++r) {
    Picture* rp;
    if ((rc = picture_of(c, f->ref_ids[r], &rp))) return rc;
    if (!rp->is_ref) return fail(c, RME_EINVAL, "reference picture was uploaded without as_ref");
    if (rp->d.codec != src->d.codec || rp->d.bit_depth != src->d.bit_depth || rp->d.width != src->d.width ||
        rp->d.height != src->d.height)
      return fail(c, RME_EINVAL, "reference format differs from the source's");
    B->ref[r] = rp->planes;
  }
  for (int i = 0; i < n; ++i) {
    const rme_bi_job& j = jobs[i];
    if (j.ref[0] < 0 || j.ref[0] >= f->nref || j.ref[1] < 0 || j.ref[1] >= f->nref || j.w < 4 || j.h < 4 ||
        j.w > 64 || j.h > 64 || (j.w & 3) || (j.h & 3) || j.x < 0 || j.y < 0 || j.x + j.w > src->cw ||
        j.y + j.h > src->ch || (refine && (j.list < 0 || j.list > 1)))
      return fail(c, RME_EINVAL, "bi job " + std::to_string(i) + " out of range");
  }
  B->width = src->cw;
  B->height = src->ch;
  B->bd = src->d.bit_depth;
  B->pad = p->hevc_pad;
  // HalfPlanes builds the quarter phases up to 2,200,000 luma samples
  // (h265_search.rs:35, 82).
  B->quarter = (int64_t)src->d.width * src->d.height <= 2200000;
  B->n = n;
  CK(cudaSetDevice(c->device));
  CK(c->d_bijobs.ensure(std::max(n, 1)));
  if (n > 0) CK(cudaMemcpyAsync(c->d_bijobs.p, jobs, sizeof(rme_bi_job) * n, cudaMemcpyHostToDevice, s));
  B->jobs = c->d_bijobs.p;
  return 0;
}
}  // namespace

int rme_bi_satd(void* ctx, const rme_frame* f, const rme_params* p, const rme_bi_job* jobs, int32_t n,
                uint32_t* satd, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (n > 0 && !satd) return fail(c, RME_EINVAL, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  BiDesc B;
  int rc = bi_setup(c, f, p, jobs, n, false, s, &B);
  if (rc || n == 0) return rc;
  CK(c->d_bisatd.ensure(n));
  CK(launch_bi_satd(B, c->d_bisatd.p, s));
  CK(cudaMemcpyAsync(satd, c->d_bisatd.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_bi_satd_weighted(void* ctx, const rme_frame* f, const rme_params* p, const rme_bi_job* jobs, int32_t n,
                         int32_t log2_wd, int32_t w0, int32_t w1, int32_t o0, int32_t o1, uint32_t* satd,
                         void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (n > 0 && !satd) return fail(c, RME_EINVAL, "null argument");
  const int lim = 1 << 12;
  if (log2_wd < 0 || log2_wd > 14 || w0 < -128 || w0 > 255 || w1 < -128 || w1 > 255 || o0 < -lim || o0 > lim ||
      o1 < -lim || o1 > lim)
    return fail(c, RME_EINVAL, "weighting out of range");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  BiDesc B;
  int rc = bi_setup(c, f, p, jobs, n, false, s, &B);
  if (rc || n == 0) return rc;
  B.wp = 1;
  B.log2_wd = log2_wd;
  B.w0 = w0;
  B.w1 = w1;
  B.o0 = o0;
  B.o1 = o1;
  CK(c->d_bisatd.ensure(n));
  CK(launch_bi_satd(B, c->d_bisatd.p, s));
  CK(cudaMemcpyAsync(satd, c->d_bisatd.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_hevc_weighted_refine(void* ctx, const rme_frame* f, const rme_params* p, int32_t log2_wd, int32_t weight,
                             int32_t offset, rme_result* out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (!f || (f->njobs > 0 && (!f->jobs || !out)) || f->njobs < 0) return fail(c, RME_EINVAL, "null argument");
  if (log2_wd < 0 || log2_wd > 14 || weight < -128 || weight > 255 || offset < -(1 << 12) || offset > (1 << 12))
    return fail(c, RME_EINVAL, "weighting out of range");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  BiDesc B;
  int rc = bi_setup(c, f, p, nullptr, 0, false, s, &B);
  if (rc) return rc;
  const int n = f->njobs;
  for (int i = 0; i < n; ++i) {
    const rme_job& j = f->jobs[i];
    if (j.ref < 0 || j.ref >= f->nref || j.nseeds < 1 || j.w < 4 || j.h < 4 || j.w > 64 || j.h > 64 || (j.w & 3) ||
        (j.h & 3) || j.x < 0 || j.y < 0 || j.x + j.w > B.width || j.y + j.h > B.height)
      return fail(c, RME_EINVAL, "job " + std::to_string(i) + " out of range");
  }
  if (n == 0) return 0;
  Picture* src;
  if ((rc = picture_of(c, f->src_id, &src))) return rc;
  const Tables* t = get_tables(c, p, src->d.bit_depth, &rc);
  if (!t) return rc;
  B.n = n;
  CK(c->d_wjobs.ensure(n));
  CK(c->d_wout.ensure(n));
  CK(cudaMemcpyAsync(c->d_wjobs.p, f->jobs, sizeof(rme_job) * n, cudaMemcpyHostToDevice, s));
  CK(launch_weighted_refine(B, c->d_wjobs.p, log2_wd, weight, offset, p->hevc_quarter_cross, t->lam, c->d_wout.p, s));
  CK(cudaMemcpyAsync(out, c->d_wout.p, sizeof(rme_result) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_bi_refine(void* ctx, const rme_frame* f, const rme_params* p, const rme_bi_job* jobs, int32_t n,
                  rme_result* out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (n > 0 && !out) return fail(c, RME_EINVAL, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  BiDesc B;
  int rc = bi_setup(c, f, p, jobs, n, true, s, &B);
  if (rc || n == 0) return rc;
  const int bps = B.bd == 8 ? 1 : 2;
  CK(c->d_bitarget.ensure((size_t)n * kBiBlock * kBiBlock * bps));
  CK(launch_bi_target(B, c->d_bitarget.p, s));
  // Each job is a GIVEN search of its list's reference from the list's own
  // vector with the job's AMVP pair, whose source is the target.
  std::vector<rme_job> gj(n);
  for (int i = 0; i < n; ++i) {
    const rme_bi_job& j = jobs[i];
    rme_job& g = gj[i];
    std::memset(&g, 0, sizeof(g));
    g.x = j.x;
    g.y = j.y;
    g.w = j.w;
    g.h = j.h;
    g.ref = j.ref[j.list];
    g.nseeds = 1;
    g.mvp[0] = j.mvp[0];
    g.mvp[1] = j.mvp[1];
    g.seeds[0] = j.mv[j.list];
  }
  rme_frame gf = *f;
  gf.jobs = gj.data();
  gf.njobs = n;
  rme_params gp = *p;
  gp.predictor_mode = RME_PRED_GIVEN;
  return run_launch(c, &gf, &gp, 1, out, nullptr, s, false, c->d_bitarget.p);
}

// ---- H.264 B pairs: b_mb's bi_refine (h264_analyse.rs:2793-2900) -------------

int rme_h264_bi_refine(void* ctx, const rme_frame* f, const rme_params* p, const rme_h264_bi_job* jobs, int32_t n,
                       int32_t rounds, int32_t diamond, rme_mv* mv_out, uint32_t* cost_out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (!f || !p || n < 0 || (n > 0 && (!jobs || !mv_out || !cost_out))) return fail(c, RME_EINVAL, "null argument");
  if (rounds < 0 || rounds > 16) return fail(c, RME_EINVAL, "rounds must be 0..16");
  Picture* src;
  int rc = picture_of(c, f->src_id, &src);
  if (rc) return rc;
  if (src->d.codec != RME_CODEC_H264) return fail(c, RME_EINVAL, "bi refinement jobs are H.264's");
  if (f->nref < 1 || f->nref > RME_MAX_REFS) return fail(c, RME_EINVAL, "nref must be 1..4");
  if ((rc = check_params(c, p, src->d))) return rc;
  DevPlanes refs[RME_MAX_REFS];
  for (int r = 0; r < f->nref; ++r) {
    Picture* rp;
    if ((rc = picture_of(c, f->ref_ids[r], &rp))) return rc;
    if (!rp->is_ref) return fail(c, RME_EINVAL, "reference picture was uploaded without as_ref");
    if (rp->d.codec != src->d.codec || rp->d.bit_depth != src->d.bit_depth || rp->d.width != src->d.width ||
        rp->d.height != src->d.height)
      return fail(c, RME_EINVAL, "reference format differs from the source's");
    refs[r] = rp->planes;
  }
  for (int i = 0; i < n; ++i) {
    const rme_h264_bi_job& j = jobs[i];
    if (j.ref[0] < 0 || j.ref[0] >= f->nref || j.ref[1] < 0 || j.ref[1] >= f->nref || j.w < 4 || j.h < 4 ||
        j.w > 16 || j.h > 16 || (j.w & 3) || (j.h & 3) || j.x < 0 || j.y < 0 || j.x + j.w > src->cw ||
        j.y + j.h > src->ch)
      return fail(c, RME_EINVAL, "bi job " + std::to_string(i) + " out of range");
    // Every vector the job can reach reads inside its search planes
    // (search_bounds, h264_hpel.rs:476-488, no vertical limit).
    const int lx = 4 - p->h264_pad - j.x, hx = src->cw + p->h264_pad - (j.w + 4) - j.x;
    const int ly = 4 - p->h264_pad - j.y, hy = src->ch + p->h264_pad - (j.h + 4) - j.y;
    for (int l = 0; l < 2; ++l)
      if (((j.mv[l].x - rounds) >> 2) < lx || ((j.mv[l].x + rounds) >> 2) >= hx ||
          ((j.mv[l].y - rounds) >> 2) < ly || ((j.mv[l].y + rounds) >> 2) >= hy)
        return fail(c, RME_EINVAL, "bi job " + std::to_string(i) + " can reach outside the search planes");
  }
  if (n == 0) return 0;
  const Tables* t = get_tables(c, p, src->d.bit_depth, &rc);
  if (!t) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  CK(c->d_h264bi.ensure((size_t)n));
  CK(c->d_bimv.ensure((size_t)2 * n));
  CK(c->d_bisatd.ensure(n));
  CK(cudaMemcpyAsync(c->d_h264bi.p, jobs, sizeof(rme_h264_bi_job) * n, cudaMemcpyHostToDevice, s));
  CK(launch_h264_bi(src->planes, refs, f->nref, src->d.bit_depth, t->tab, c->d_h264bi.p, n, rounds, diamond ? 4 : 8,
                    c->d_bimv.p, c->d_bisatd.p, s));
  CK(cudaMemcpyAsync(mv_out, c->d_bimv.p, sizeof(rme_mv) * 2 * n, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(cost_out, c->d_bisatd.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_chroma_predict(void* ctx, int32_t ref_id, int32_t nblocks, const int32_t* blocks, const rme_mv* mvs,
                       void* out, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  Picture* p;
  int rc = picture_of(c, ref_id, &p);
  if (rc) return rc;
  if (!p->chroma) return fail(c, RME_EINVAL, "no chroma uploaded for this picture");
  if (nblocks < 0 || (nblocks > 0 && (!blocks || !mvs || !out))) return fail(c, RME_EINVAL, "bad block list");
  if (nblocks == 0) return 0;
  std::vector<int64_t> off(nblocks);
  int64_t total = 0;
  for (int i = 0; i < nblocks; ++i) {
    const int32_t* b = blocks + 4 * i;
    if (b[0] < 0 || b[1] < 0 || b[2] < 2 || b[3] < 2 || b[2] > 128 || b[3] > 128 || b[0] + b[2] > p->d.width ||
        b[1] + b[3] > p->d.height)
      return fail(c, RME_EINVAL, "block " + std::to_string(i) + " outside the picture");
    off[i] = total;
    total += 2 * (int64_t)(b[2] / 2) * (b[3] / 2);
  }
  const int bps = p->d.bit_depth == 8 ? 1 : 2;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  cudaPointerAttributes pa{};
  const bool dev_out = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeDevice;
  cudaGetLastError();
  CK(c->d_cblk.ensure(4 * (int64_t)nblocks));
  CK(c->d_cmv.ensure(nblocks));
  CK(c->d_coff.ensure(nblocks));
  if (!dev_out) CK(c->d_cout.ensure(total * bps));
  CK(cudaMemcpyAsync(c->d_cblk.p, blocks, sizeof(int32_t) * 4 * nblocks, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(c->d_cmv.p, mvs, sizeof(rme_mv) * nblocks, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(c->d_coff.p, off.data(), sizeof(int64_t) * nblocks, cudaMemcpyHostToDevice, s));
  const int cw = p->d.width / 2, ch = p->d.height / 2;
  const uint8_t* cb = (const uint8_t*)p->chroma;
  const uint8_t* cr = cb + (size_t)cw * ch * bps;
  void* dst = dev_out ? out : (void*)c->d_cout.p;
  CK(launch_chroma(cb, cr, p->d.bit_depth, p->d.codec, cw, ch, cw, nblocks, c->d_cblk.p, c->d_cmv.p, c->d_coff.p, dst,
                   s));
  if (!dev_out) CK(cudaMemcpyAsync(out, c->d_cout.p, (size_t)total * bps, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

namespace {
bool device_accessible(const void* ptr, int* dev) {
  cudaPointerAttributes pa{};
  const bool ok = ptr && cudaPointerGetAttributes(&pa, ptr) == cudaSuccess &&
                  (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  if (ok && dev) *dev = pa.device;
  return ok;
}

int dist_batch(bool satd, const void* a, int64_t as, const int64_t* aoff, const void* b, int64_t bs,
               const int64_t* boff, int32_t w, int32_t h, int32_t bd, int32_t n, uint32_t* out, void* stream) {
  if (n < 0 || w < 1 || h < 1 || w > 256 || h > 256 || bd < 8 || bd > 14 || as < w || bs < w) return RME_EINVAL;
  if (satd && ((w & 3) || (h & 3))) return RME_EINVAL;
  if (n == 0) return 0;
  int dev = 0;
  if (!device_accessible(a, &dev) || !device_accessible(b, nullptr) || !device_accessible(aoff, nullptr) ||
      !device_accessible(boff, nullptr) || !device_accessible(out, nullptr))
    return RME_EINVAL;
  if (cudaSetDevice(dev) != cudaSuccess) return RME_ECUDA;
  return launch_dist_batch(satd, a, as, aoff, b, bs, boff, w, h, bd, n, out, (cudaStream_t)stream) == cudaSuccess
             ? 0
             : RME_ECUDA;
}
}  // namespace

int rme_sad_batch(const void* a, int64_t a_stride, const int64_t* a_off, const void* b, int64_t b_stride,
                  const int64_t* b_off, int32_t w, int32_t h, int32_t bit_depth, int32_t n, uint32_t* out,
                  void* stream) {
  return dist_batch(false, a, a_stride, a_off, b, b_stride, b_off, w, h, bit_depth, n, out, stream);
}
int rme_satd_batch(const void* a, int64_t a_stride, const int64_t* a_off, const void* b, int64_t b_stride,
                   const int64_t* b_off, int32_t w, int32_t h, int32_t bit_depth, int32_t n, uint32_t* out,
                   void* stream) {
  return dist_batch(true, a, a_stride, a_off, b, b_stride, b_off, w, h, bit_depth, n, out, stream);
}

// ---- lookahead at half resolution (h265_cutree.rs, h264_lookahead.rs) --------

int rme_lowres_build(void* ctx, int32_t pic_id, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  Picture* p;
  int rc = picture_of(c, pic_id, &p);
  if (rc) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  LowresDesc L{};
  L.h264 = p->d.codec == RME_CODEC_H264;
  if (L.h264) {
    // One 8x8 block per macroblock (h264_lookahead.rs:87-117).
    L.bw = (p->d.width + 15) / 16;
    L.bh = (p->d.height + 15) / 16;
    L.bytes = p->d.bit_depth > 8 ? 2 : 1;
  } else {
    const int lw = (p->d.width + 1) / 2, lh = (p->d.height + 1) / 2;
    L.bw = (lw + 7) / 8;
    L.bh = (lh + 7) / 8;
    L.bytes = 1;
  }
  L.pw = L.bw * 8;
  L.ph = L.bh * 8;
  L.stride = L.pw + 2 * kLowresPad;
  const size_t plane = (size_t)L.stride * (L.ph + 2 * kLowresPad) * L.bytes,
               intra = sizeof(uint32_t) * L.bw * L.bh;
  if (!p->lowres) CK(cudaMalloc(&p->lowres, plane + 256 + intra));
  L.plane = (uint8_t*)p->lowres;
  L.intra = (uint32_t*)((uint8_t*)p->lowres + (plane + 255) / 256 * 256);
  p->lr = L;
  CK(launch_lowres_build(p->planes, p->d.bit_depth, p->d.width, p->d.height, L, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int rme_lowres_info(void* ctx, int32_t pic_id, int32_t* bw, int32_t* bh, uint32_t* intra) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  Picture* p;
  int rc = picture_of(c, pic_id, &p);
  if (rc) return rc;
  if (!p->lowres) return fail(c, RME_EINVAL, "no half-resolution plane: call rme_lowres_build");
  if (bw) *bw = p->lr.bw;
  if (bh) *bh = p->lr.bh;
  if (intra) CK(cudaMemcpy(intra, p->lr.intra, sizeof(uint32_t) * p->lr.bw * p->lr.bh, cudaMemcpyDeviceToHost));
  return 0;
}

namespace {
int lowres_pair(Ctx* c, int32_t a, int32_t b, Picture** pa, Picture** pb) {
  int rc = picture_of(c, a, pa);
  if (!rc) rc = picture_of(c, b, pb);
  if (rc) return rc;
  if (!(*pa)->lowres || !(*pb)->lowres) return fail(c, RME_EINVAL, "no half-resolution plane: call rme_lowres_build");
  if ((*pa)->lr.bw != (*pb)->lr.bw || (*pa)->lr.bh != (*pb)->lr.bh || (*pa)->lr.h264 != (*pb)->lr.h264 ||
      (*pa)->lr.bytes != (*pb)->lr.bytes)
    return fail(c, RME_EINVAL, "half-resolution sizes differ");
  return 0;
}
}  // namespace

int rme_lowres_search_batch(void* ctx, int32_t npairs, const int32_t* cur_ids, const int32_t* ref_ids, uint32_t* cost,
                            rme_mv* mv, uint32_t* nsad, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (npairs < 1 || !cur_ids || !ref_ids || !cost || !mv) return fail(c, RME_EINVAL, "null argument");
  std::vector<LowresDesc> pairs(2 * (size_t)npairs);
  for (int k = 0; k < npairs; ++k) {
    Picture *pc, *pr;
    int rc = lowres_pair(c, cur_ids[k], ref_ids[k], &pc, &pr);
    if (rc) return rc;
    pairs[2 * k] = pc->lr;
    pairs[2 * k + 1] = pr->lr;
    const LowresDesc &a = pairs[0], &b = pc->lr;
    if (b.bw != a.bw || b.bh != a.bh || b.h264 != a.h264 || b.bytes != a.bytes)
      return fail(c, RME_EINVAL, "the pairs' half-resolution formats differ");
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  const int bw = pairs[0].bw, bh = pairs[0].bh, n = bw * bh;
  const int64_t total = (int64_t)n * npairs;
  // Claim order: anti-diagonals, each block after its left and above ones.
  if (c->lorder_shape != std::make_pair(bw, bh)) {
    std::vector<int32_t> order;
    order.reserve(n);
    for (int d = 0; d <= bw + bh - 2; ++d)
      for (int by = std::max(0, d - bw + 1); by <= std::min(d, bh - 1); ++by) order.push_back((by << 16) | (d - by));
    CK(c->d_lorder.ensure(n));
    CK(cudaMemcpy(c->d_lorder.p, order.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    c->lorder_shape = {bw, bh};
  }
  CK(c->d_ldone.ensure(total + 8));
  CK(c->d_lcost.ensure(total));
  CK(c->d_lsad.ensure(total));
  CK(c->d_lmv.ensure(total));
  CK(c->d_lpairs.ensure(2 * (int64_t)npairs));
  CK(cudaMemcpyAsync(c->d_lpairs.p, pairs.data(), sizeof(LowresDesc) * pairs.size(), cudaMemcpyHostToDevice, s));
  // done flags, then the claim counter and the status word (one memset).
  CK(cudaMemsetAsync(c->d_ldone.p, 0, sizeof(int32_t) * (total + 8), s));
  const int64_t ci = (total + 3) & ~int64_t(1);  // an 8-byte aligned word after the flags
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(c->d_ldone.p + ci);
  uint32_t* status = reinterpret_cast<uint32_t*>(c->d_ldone.p + ci + 2);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(c->nsm * 4, (total + 7) / 8));
  CK(launch_lowres_search(c->d_lpairs.p, npairs, pairs[0], c->d_lorder.p, c->d_ldone.p, counter, status, c->d_lcost.p,
                          c->d_lmv.p, c->d_lsad.p, grid, s));
  uint32_t st = 0;
  CK(cudaMemcpyAsync(cost, c->d_lcost.p, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(mv, c->d_lmv.p, sizeof(rme_mv) * total, cudaMemcpyDeviceToHost, s));
  if (nsad) CK(cudaMemcpyAsync(nsad, c->d_lsad.p, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&st, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (st) return fail(c, RME_EDEVICE, "device status " + std::to_string(st));
  return 0;
}

int rme_lowres_search(void* ctx, int32_t cur_id, int32_t ref_id, uint32_t* cost, rme_mv* mv, uint32_t* nsad,
                      void* stream) {
  return rme_lowres_search_batch(ctx, 1, &cur_id, &ref_id, cost, mv, nsad, stream);
}

int rme_lowres_bi_cost(void* ctx, int32_t cur_id, int32_t r0_id, const rme_mv* mv0, int32_t r1_id, const rme_mv* mv1,
                       uint32_t* cost, void* stream) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return RME_EINVAL;
  if (!mv0 || !mv1 || !cost) return fail(c, RME_EINVAL, "null argument");
  Picture *pc, *p0, *p1;
  int rc = lowres_pair(c, cur_id, r0_id, &pc, &p0);
  if (!rc) rc = lowres_pair(c, cur_id, r1_id, &pc, &p1);
  if (rc) return rc;
  const int n = pc->lr.bw * pc->lr.bh;
  // Every displaced block must stay in the padded plane (the search's own
  // vectors always do).
  for (int i = 0; i < n; ++i) {
    const int x = (i % pc->lr.bw) * 8, y = (i / pc->lr.bw) * 8;
    for (const rme_mv* m : {mv0 + i, mv1 + i})
      if (x + m->x < -kLowresPad || y + m->y < -kLowresPad || x + m->x + 8 > pc->lr.pw + kLowresPad ||
          y + m->y + 8 > pc->lr.ph + kLowresPad)
        return fail(c, RME_EINVAL, "vector of block " + std::to_string(i) + " leaves the padded plane");
  }
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  CK(cudaSetDevice(c->device));
  CK(c->d_lmv.ensure(n));
  CK(c->d_lmv2.ensure(n));
  CK(c->d_lcost.ensure(n));
  CK(cudaMemcpyAsync(c->d_lmv.p, mv0, sizeof(rme_mv) * n, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(c->d_lmv2.p, mv1, sizeof(rme_mv) * n, cudaMemcpyHostToDevice, s));
  CK(launch_lowres_bi(pc->lr, p0->lr, p1->lr, c->d_lmv.p, c->d_lmv2.p, c->d_lcost.p, s));
  CK(cudaMemcpyAsync(cost, c->d_lcost.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

}  // extern "C"
