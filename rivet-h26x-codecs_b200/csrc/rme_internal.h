// Internal structures shared by the host side (rme_capi.cu) and the kernels
// (rme_planes.cu, rme_search.cu) of librivet_me.so. Not part of the ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rivet_me.h"

namespace rme {

constexpr int kH264Pad = 32;  // h264/frame.rs LUMA_PAD
constexpr int kHevcPad = 80;  // hevc/frame.rs LUMA_PAD
constexpr int kChromaPadHevc = 40;
constexpr int kChromaPadH264 = 16;
constexpr int kMvSpan = 4096;  // h264_hpel.rs MV_SPAN
constexpr int kMvTab = 2 * kMvSpan + 1;
constexpr int kMaxLevels = 4;
constexpr int kWarpsPerBlock = 8;
constexpr uint32_t kSpinLimit = 1u << 22;  // bounded dependency waits

// Device status word bits.
constexpr uint32_t kStatusWaitTimeout = 1u;
constexpr uint32_t kStatusBadTask = 2u;
constexpr uint32_t kStatusBounds = 4u;

// One picture's planes on the device: `nplanes` planes of rows x stride
// samples, one allocation; `origin` is the offset of visible sample (0, 0)
// within a plane. H.264 pictures hold G, b, h, j; HEVC pictures hold G and
// the 15 fractional phases (index fy*4+fx).
struct DevPlanes {
  const void* base;
  int64_t plane_elems;
  int32_t stride;
  int32_t origin;
};

// One frame of a launch, as the kernel reads it.
struct FrameDesc {
  int32_t codec, bd, mode, nref;
  int32_t width, height;  // H.264: the coded (macroblock-rounded) size
  int32_t pad;            // the reference's plane border (search semantics)
  DevPlanes src;
  DevPlanes ref[RME_MAX_REFS];
  // HEVC
  int32_t nlevels;
  int32_t size[kMaxLevels], nbx[kMaxLevels], nby[kMaxLevels], base[kMaxLevels + 1];
  int32_t search_range, search_rings, quarter_cross;
  float lam;                 // SATD Lagrangian (rate = (lam * bits as f32) as u32)
  // STANDALONE AMP: mode bits, their count, the levels that have AMP units
  // (the first amp_nlev: sizes of 16 or more), and per such level the block
  // index of its first AMP unit (amp_base[0] = base[nlevels]).
  int32_t amp, amp_nmodes, amp_nlev;
  int32_t amp_base[kMaxLevels + 1];
  // H.264
  const uint16_t* tab;       // MvCostTable
  int32_t range, hpel_iters, qpel_iters, umh, qpel_diamond, dia, vr;
  float refine_ratio;
  uint32_t ref_cost[RME_MAX_REFS];
  // GIVEN
  const rme_job* jobs;
  // GIVEN, HEVC refine_bi: per task its source block (the bi target),
  // kBiBlock x kBiBlock samples at t * kBiBlock^2, searched at 2 * lam.
  const void* bi_src;
  // outputs, and per task the count of its unfinished dependencies
  rme_result* out;
  int32_t* pending;
  int32_t ntasks;
  uint32_t gen;  // the resident engine: this frame's generation in its slot
  int32_t big_end;  // HEVC STANDALONE: tasks below big_end * nref are blocks of 32 or more
  // The row form (HEVC STANDALONE without AMP, latency kernels and the
  // engine): a warp or a CTA owns a row of one level and reference and
  // searches its blocks left to right; per task its motion vector is
  // published as one word, (tag << 32) | mv, which the rows below and the
  // next size's rows wait for. Null: the dataflow form.
  unsigned long long* mvf;
  uint32_t tag;     // nonzero, new for every search of the buffer (the launch's epoch, the slot's generation)
  int32_t nrows;    // rows of the frame, both kinds (the engine counts them to completion)
};

// A row-form queue entry's low 24 bits: level (bits 22-23), reference
// (20-21), row (0-19).
constexpr uint32_t row_entry(int l, int r, int row) { return (uint32_t)l << 22 | (uint32_t)r << 20 | (uint32_t)row; }

// A launch's dataflow queue: a task is pushed when its last dependency
// finishes (the frames' dependency-free tasks are pushed by the host), and
// warps pop in push order. Slots hold (epoch << 32) | (frame << 24) | task,
// so a slot of an earlier launch never reads as filled.
struct LaunchDesc {
  const FrameDesc* frames;
  unsigned long long* ready;     // capacity `total`
  int64_t total;                 // tasks of this launch (= pushes = pops)
  unsigned long long* head;      // next slot to pop
  unsigned long long* tail;      // next slot to push (starts at the host's count)
  uint32_t* status;
  unsigned long long* counters;  // [tasks, sad, satd, sad_samples, satd_samples]
  const uint32_t* epoch;         // this launch's epoch (device memory: a
                                 // replayed graph keeps its arguments)
  unsigned long long* done;      // tasks finished, or null: with it a warp
                                 // runs one task it made ready itself
                                 // (no queue round trip) and idle warps
                                 // leave once every task is done
  // The queue of the tasks a whole CTA runs (32x32 and 64x64 blocks in the
  // latency form), served by the first `group_ctas` CTAs; 0: none.
  unsigned long long* ready_big;
  unsigned long long* head_big;
  unsigned long long* tail_big;
  int32_t group_ctas;
  int32_t patch8;                // the latency form: 8x8 blocks refine from staged phase patches
  int32_t ring_shift;            // nonzero: the resident engine's ring of
                                 // 2^ring_shift slots (ring_entry)
  int32_t rows;                  // the row form: the queues hold rows, all pushed by the host
  int64_t total_big;             // the row form: rows in the CTAs' queue
};

// The resident engine (rme_engine.cu): one search kernel that stays on the
// GPU while a serving loop feeds it frames of any kind. Frames occupy slots
// of a device table; a frame's tasks enter the ring as its planes are built;
// the warp that finishes a frame's last task raises the frame's flag in
// mapped host memory.
constexpr int kEngineFrames = 256;  // frame slots (the queue's 8-bit frame field)
struct EngineCtl {
  uint32_t* fdone;                 // per frame slot: its tasks finished
  volatile uint32_t* hflags;       // mapped host memory: per slot, the generation finished
  const uint32_t* stop;            // device memory: nonzero once waiting warps are to leave
  uint32_t idle_polls;             // reserved
};
cudaError_t launch_engine(const LaunchDesc& L, const EngineCtl& E, int grid, cudaStream_t s);
int engine_blocks_per_sm();
cudaError_t launch_publish(const LaunchDesc& L, int frame, const uint32_t* roots, int nroots, cudaStream_t s);
// The host side (one engine per context, driven by one thread): a frame is
// submitted behind its uploads on `upload` and takes a slot; engine_done
// tells when its results (engine_results, device memory) are complete;
// engine_release frees the slot once they have been copied out.
struct Engine;
int engine_create(void* ctx, int device, Engine** out);
void engine_destroy(Engine* g);
int engine_submit(Engine* g, const rme_frame* f, const rme_params* p, cudaStream_t upload, int* slot);
bool engine_done(Engine* g, int slot);
int engine_keep_running(Engine* g);
bool engine_idle(Engine* g);
int engine_stop(Engine* g);
const rme_result* engine_results(Engine* g, int slot);
int engine_slot_tasks(Engine* g, int slot);
const uint32_t* engine_status_word(Engine* g);
void engine_release(Engine* g, int slot);
// rme_capi.cu: a STANDALONE frame's descriptor over a context's pictures,
// its task count, dependency template and root tasks (device memory).
int ctx_standalone_frame(void* ctx, const rme_frame* f, const rme_params* p, FrameDesc* fd, int* ntasks,
                         const int32_t** pending_tmpl, const uint32_t** roots, int* nroots);
// rme_picture_upload with the choice to leave a reference picture's
// interpolated planes for a later rme_picture_build_planes on the same
// stream (the serving loop publishes the picture's own search first: it
// reads only the integer plane).
int ctx_picture_upload(void* ctx, int32_t pic_id, const rme_picture_desc* d, const void* luma, int32_t as_ref,
                       bool build_planes, void* stream);
// The same frame's rows (row_entry; device memory) when it can run in the
// row form: rows a warp runs, then rows a CTA runs, each in the order every
// row comes after the rows it reads. False for other frames.
bool ctx_frame_rows(void* ctx, const rme_frame* f, const rme_params* p, const uint32_t** rows, int* nrows,
                    const uint32_t** rows_big, int* nrows_big);

// Host helpers shared by the entry points (rme_capi.cu; f32 arithmetic
// compiled without contraction, so it rounds as the reference's Rust does).
float h264_mvd_bits(int d);                  // h264_hpel.rs:407-429
float h264_lambda_satd(int qp);              // h264_analyse.rs:402-404
float hevc_lambda(int qp, int bd, float scale);  // h265_intra.rs:1141-2013
void h264_cost_table(float lam, uint16_t* tab);  // kMvTab entries, MvCostTable::new
// Why a parameter block cannot be searched for a picture of `d`'s format,
// or null when it can.
const char* param_error(const rme_params* p, const rme_picture_desc& d);

// The kernels that run beside a resident search (the uploads' plane builds,
// the engine's publish) and the search kernels ask for one shared-memory
// carveout, the most shared memory: an SM's carveout is fixed while blocks
// run on it, so a kernel preferring another one waits for the SM to empty,
// which a resident search never does.
template <class K>
inline cudaError_t prefer_max_shared(K* kernel) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                              (int)cudaSharedmemCarveoutMaxShared);
}

// Launch wrappers (defined in the .cu files).
cudaError_t launch_pad_plane(const void* src, int bd, int w, int h, int sstride, DevPlanes dst, int cw, int ch,
                             int pad, cudaStream_t s);
cudaError_t launch_h264_hpel(DevPlanes p, int bd, int cw, int ch, int pad, cudaStream_t s);
cudaError_t launch_hevc_phases(DevPlanes p, int bd, int w, int h, int pad, cudaStream_t s);
// Weighted prediction (rme_wp.cu): the weighted copy of a padded plane
// (`bytes`, a multiple of 16), and the fit's passes over a picture pair
// (pointers at the visible origin, `stride` samples per row).
cudaError_t launch_weighted_plane(const void* src, void* dst, int64_t bytes, int codec, int bd, int log_wd, int weight,
                                  int offset, cudaStream_t s);
cudaError_t launch_wp_moments(const void* cur, const void* ref, int stride, int bd, int w, int h,
                              unsigned long long* out, cudaStream_t s);
cudaError_t launch_weighted_sad(const void* cur, const void* ref, int stride, int bd, int w, int h, int weight,
                                int shift, int offset, unsigned long long* out, cudaStream_t s);
// A bounded dependency wait that runs out (rme_lookahead.cu's wait on a flag
// nothing sets, `limit` polls): sets kStatusWaitTimeout in *status.
cudaError_t launch_probe_wait(const int32_t* flag, uint32_t limit, uint32_t* status, cudaStream_t s);
// HEVC bi-prediction (rme_bi.cu): the jobs of a frame's source and
// references; refine_bi targets are kBiBlock-wide blocks.
constexpr int kBiBlock = 64;
struct BiDesc {
  DevPlanes src;
  DevPlanes ref[RME_MAX_REFS];
  int32_t width, height, bd, pad, quarter;
  const rme_bi_job* jobs;
  int32_t n;
  // Explicit weighting of the bi score (wp != 0): weighted_bi's log2WD,
  // the two lists' weights and offsets.
  int32_t wp, log2_wd, w0, w1, o0, o1;
};
cudaError_t launch_bi_satd(const BiDesc& B, uint32_t* satd, cudaStream_t s);
cudaError_t launch_bi_target(const BiDesc& B, void* target, cudaStream_t s);
// HEVC weighted lists' refine_subpel (rme_bi.cu): B's jobs unused, `jobs`
// GIVEN jobs (start = seeds[0]), one result per job into `out`.
cudaError_t launch_weighted_refine(const BiDesc& B, const rme_job* jobs, int log2_wd, int weight, int offset,
                                   int quarter_cross, float lam, rme_result* out, cudaStream_t s);
// H.264 B pairs' joint refinement (rme_bi.cu): `tab` the MvCostTable.
cudaError_t launch_h264_bi(const DevPlanes& src, const DevPlanes* refs, int nref, int bd, const uint16_t* tab,
                           const rme_h264_bi_job* jobs, int n, int rounds, int npts, rme_mv* mv_out,
                           uint32_t* cost_out, cudaStream_t s);

// The lookahead's half-resolution plane of a picture, whole 8x8 blocks
// (pw x ph) padded by kLowresPad on every side: HEVC's cutree plane
// (h265_cutree.rs LowRes, 8-bit) or H.264's lookahead plane
// (h264_lookahead.rs, the stream's sample type, one block per macroblock).
constexpr int kLowresPad = 24, kLowresRange = 16;
struct LowresDesc {
  uint8_t* plane;   // (ph + 2 pad) rows of `stride` samples of `bytes` bytes
  uint32_t* intra;  // per block, raster
  int32_t stride, pw, ph, bw, bh;
  int32_t h264, bytes;
};
cudaError_t launch_lowres_build(const DevPlanes& pic, int bd, int w, int h, const LowresDesc& L, cudaStream_t s);
// `pairs`: device array of (cur, ref) descriptors of npairs pairs that share
// the block grid of `first`; per-pair outputs and done flags npairs x blocks.
cudaError_t launch_lowres_search(const LowresDesc* pairs, int npairs, const LowresDesc& first, const int32_t* order,
                                 int32_t* done, unsigned long long* counter, uint32_t* status, uint32_t* cost,
                                 rme_mv* mv, uint32_t* nsad, int grid, cudaStream_t s);
cudaError_t launch_lowres_bi(const LowresDesc& cur, const LowresDesc& r0, const LowresDesc& r1, const rme_mv* m0,
                             const rme_mv* m1, uint32_t* cost, cudaStream_t s);

// The search over one kind of task (sample width, codec): `grid` persistent
// blocks pulling from L's queue. `variant` picks the kernel's occupancy
// bound: 0, 1, 2 for 2, 3, 4 resident blocks per SM (1 is the default).
constexpr int kSearchVariants = 3, kDefaultVariant = 1;
// `spec` picks the latency form (HEVC: 8x8 diamonds two rounds per step)
// for launches of a frame or two; results are the same.
cudaError_t launch_search(const LaunchDesc& L, int bytes_per_sample, int codec, int variant, int grid,
                          cudaStream_t s, bool spec = false);
int search_blocks_per_sm(int bytes_per_sample, int codec, int variant, bool spec = false);
cudaError_t launch_chroma(const void* cb, const void* cr, int bd, int codec, int cw, int ch, int cstride,
                          int nblocks, const int32_t* blocks, const rme_mv* mvs, const int64_t* out_off, void* out,
                          cudaStream_t s);
cudaError_t launch_dist_batch(bool satd, const void* a, int64_t as, const int64_t* aoff, const void* b, int64_t bs,
                              const int64_t* boff, int w, int h, int bd, int n, uint32_t* out, cudaStream_t s);

}  // namespace rme
