/*
 * rivet_me.h — C ABI of the B200 motion-estimation library (librivet_me.so).
 *
 * The library replaces the motion-search stage of the rivet-h26x encoders:
 *   H.264  Search::int_search / Search::refine        src/encode/h264_hpel.rs:789-1021
 *          (driven per macroblock by p_mb)            src/encode/h264_analyse.rs:1884-1975
 *   HEVC   InterPicture::search_full / refine_subpel  src/encode/h265_me.rs:3749-3922
 *          (driven per prediction unit by pick_pu)    src/encode/h265_me.rs:1327-1380
 * together with the per-reference plane builds they read
 *   H.264  build_hpel / hpel_planes                   src/encode/h264_hpel.rs:95-189
 *   HEVC   HalfPlanes::new                            src/encode/h265_search.rs:79-170
 * and the DSP kernels underneath (dsp/distortion.rs sad/satd, dsp/hevc.rs
 * qpel_h/v/v2, epel_h/v/v2, uni, dsp/h264.rs qpel/chroma).
 *
 * The reference calls one scalar/SIMD kernel per candidate through plain
 * function pointers (DistortionDsp, HevcDsp, H264EncDsp). A GPU launch per
 * candidate would cost more than the candidate, so this boundary is
 * batched: a caller uploads pictures once, then submits whole frames (or
 * lists of prediction-unit jobs), and reads back one result per job.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative RME_E* code; the
 *    text of the last error of a context is rme_last_error(). No function
 *    aborts or throws across the ABI.
 *  - Motion vectors are quarter-sample int16 pairs, as rivet's Mv.
 *  - Pictures are passed unpadded, row-major, `stride` samples per row;
 *    8-bit pictures are uint8_t, deeper ones uint16_t (Sample = u8 | u16,
 *    src/sample.rs:7-56). The library pads them on the device by edge
 *    replication, which is what the reference's padded planes hold
 *    (hevc/frame.rs:317-340 extend_rows, h264/frame.rs extend_edges).
 *  - A context is bound to one CUDA device; calls on one context must not
 *    overlap from several host threads. Separate contexts are independent.
 *  - `stream` arguments are cudaStream_t passed as void* (0 = the legacy
 *    default stream), so this header needs no CUDA include.
 */
#ifndef RIVET_ME_H
#define RIVET_ME_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------- */
#define RME_OK             0
#define RME_EINVAL        -1   /* bad argument (size, depth, id, pointer)   */
#define RME_ENOMEM        -2   /* device or host allocation failed           */
#define RME_ECUDA         -3   /* a CUDA call failed (text in last_error)    */
#define RME_ENOTFOUND     -4   /* picture id not uploaded                    */
#define RME_EDEVICE       -5   /* device status word set: a bounded wait ran
                                  out or a bounds check fired in a kernel    */
#define RME_EBUSY         -6   /* admission refused (budget / queue full)    */
#define RME_ENOSYS        -7   /* not built for this configuration          */

/* ---- enums -------------------------------------------------------------- */
#define RME_CODEC_H264     0
#define RME_CODEC_HEVC     1

/* How prediction-unit seeds and predictors are supplied.
 * GIVEN:      the caller passes one rme_job per (block, reference) with its
 *             predictor(s) and candidate seeds — one encoder call exactly.
 * STANDALONE: the library derives them from the frame's own results in a
 *             fixed order (a wavefront): HEVC, per reference and size
 *             level, the AMVP pair of the left and upper blocks' results
 *             and the enclosing block's result as the parent seed; H.264,
 *             p_mb's candidates over the A, B, C, D macroblocks' results.
 *             Used for whole-frame throughput runs.                      */
#define RME_PRED_GIVEN       0
#define RME_PRED_STANDALONE  1

/* H.264 GIVEN-mode job flags */
#define RME_JOB_SCORE_ONLY   1  /* refine with MeCfg::SCORE (score the whole-
                                   sample winner, no sub-sample rounds):
                                   p_mb's refine_ratio branch             */

#define RME_MAX_SEEDS        10 /* 3 + MAX_MERGE_CAND + 1 (h265_me.rs:1327) */
#define RME_MAX_REFS         4

typedef struct { int16_t x, y; } rme_mv;

/* A picture as the caller holds it. */
typedef struct {
  int32_t codec;      /* RME_CODEC_*                                        */
  int32_t bit_depth;  /* 8 (uint8_t samples) or 9..12 (uint16_t samples)   */
  int32_t width;      /* luma width and height in samples                  */
  int32_t height;
  int32_t stride;     /* luma row stride of the host buffer, in samples     */
} rme_picture_desc;

/* Search settings: the reference's MeCfg / AnalysisCfg (H.264) and the
 * h265_me constants / Tune knobs (HEVC). rme_params_default() fills the
 * reference's medium tier. */
typedef struct {
  int32_t codec;
  int32_t qp;
  int32_t predictor_mode;     /* RME_PRED_*                                 */
  /* H.264: MeCfg (h264_hpel.rs:492-519) of AnalysisCfg::me              */
  int32_t h264_range;
  int32_t h264_hpel_iters;
  int32_t h264_qpel_iters;
  int32_t h264_umh;
  int32_t h264_qpel_diamond;
  int32_t h264_dia;
  float   h264_refine_ratio;  /* AnalysisCfg::refine_ratio (0: always)      */
  int32_t h264_vertical_range;/* MotionLimits::vertical_search, full samples */
  int32_t h264_pad;           /* search plane border, h264/frame.rs LUMA_PAD */
  /* HEVC: h265_me.rs SEARCH_RANGE, Tune::search_rings / quarter_cross,
   * Tune::lambda (P pictures), hevc/frame.rs LUMA_PAD                    */
  int32_t hevc_search_range;
  int32_t hevc_search_rings;
  int32_t hevc_quarter_cross;
  float   hevc_lambda_scale;
  int32_t hevc_pad;
  int32_t hevc_pu_mask;       /* STANDALONE: bit k -> 2Nx2N PUs of 8<<k     */
  int32_t hevc_amp;           /* STANDALONE: also the AMP units of every
                                 CU of size >= 16: bit 0 2NxnU, 1 2NxnD,
                                 2 nLx2N, 3 nRx2N (each CU's two units,
                                 searched from the CU's 2Nx2N result)      */
} rme_params;

/* One search job (GIVEN mode): a block, the reference it searches, its
 * predictor(s) and seeds, in the order the encoder assembles them.
 *  HEVC : mvp = the two AMVP predictors of this reference; seeds as pick_pu
 *         builds them (zero, mvp0, mvp1, merge vectors of this ref,
 *         parent seed).
 *  H.264: mvp[0] = the rate predictor (Search::pred); seeds = int_search's
 *         candidate list (p_mb: skip_mv, zero, neighbour vectors...).   */
typedef struct {
  int32_t x, y;        /* block position in luma samples                   */
  int32_t w, h;        /* block size                                        */
  int32_t ref;         /* index into the frame's reference list             */
  int32_t nseeds;      /* 0..RME_MAX_SEEDS                                  */
  int32_t flags;       /* RME_JOB_*                                         */
  rme_mv  mvp[2];
  rme_mv  seeds[RME_MAX_SEEDS];
} rme_job;

/* One search result. */
typedef struct {
  rme_mv   mv;         /* chosen quarter-sample vector                      */
  int32_t  ref;        /* its reference index                               */
  uint32_t cost;       /* SATD + rate of mv (H.264 STANDALONE: + ref bits)  */
  uint32_t satd;       /* SATD of mv, no rate                               */
  rme_mv   int_mv;     /* whole-sample stage winner                         */
  uint32_t int_cost;   /* its SAD + rate                                    */
  uint32_t n_sad;      /* SAD candidates scored (the reference's count)     */
  uint32_t n_satd;     /* SATD candidates scored                            */
} rme_result;

/* A frame of work: the source picture, its references (most recent first,
 * the order of refs_l0), the settings, and — in GIVEN mode — the jobs.   */
typedef struct {
  int32_t src_id;
  int32_t nref;
  int32_t ref_ids[RME_MAX_REFS];
  const rme_job* jobs;       /* GIVEN mode; host memory; NULL otherwise     */
  int32_t njobs;
} rme_frame;

/* Device-resident performance counters of the last completed call. */
typedef struct {
  uint64_t tasks;            /* (block, reference) searches run             */
  uint64_t sad_candidates;   /* sum of n_sad                                */
  uint64_t satd_candidates;  /* sum of n_satd                               */
  uint64_t sad_samples;      /* sum over SAD candidates of w*h              */
  uint64_t satd_samples;     /* sum over SATD candidates of w*h             */
  float    kernel_ms;        /* device time of the search launch(es)        */
  float    planes_ms;        /* device time from the first upload since the
                                previous search to the end of the last one  */
} rme_stats;

/* ---- lifecycle ---------------------------------------------------------- */

/* Medium-tier settings of `codec` at `qp`: MeCfg MEDIUM with refine_ratio
 * 1.5 (h264_analyse.rs:193-240), SEARCH_RANGE 48, no rings, the square
 * quarter ring, Tune::lambda 0.85 (h265_tune.rs:411), 2Nx2N PUs 8..64. */
void rme_params_default(rme_params* p, int32_t codec, int32_t qp);

int  rme_ctx_create(void** ctx, int32_t device);
void rme_ctx_destroy(void* ctx);
const char* rme_last_error(void* ctx);

/* ---- pictures ------------------------------------------------------------ */

/* Upload a luma picture under `pic_id` (any non-negative id; re-uploading an
 * id replaces it). `as_ref` != 0 also builds its search planes on the
 * device: the padded integer plane plus H.264's three half-sample planes
 * (b, h, j) or HEVC's fifteen fractional phases — what build_hpel and
 * HalfPlanes::new compute on the CPU. Asynchronous on `stream`; `luma` may
 * be reused once the stream has passed the call. */
int rme_picture_upload(void* ctx, int32_t pic_id, const rme_picture_desc* d,
                       const void* luma, int32_t as_ref, void* stream);

/* Upload the two chroma planes of a 4:2:0 picture (width/2 x height/2,
 * `cstride` samples per row) for rme_chroma_predict. */
int rme_picture_upload_chroma(void* ctx, int32_t pic_id, const void* cb,
                              const void* cr, int32_t cstride, void* stream);

int rme_picture_release(void* ctx, int32_t pic_id);

/* Rebuild the search planes of an uploaded reference from its resident
 * integer plane, on `stream`, without waiting: the per-reference plane
 * build (build_hpel / HalfPlanes::new) of a picture already in HBM. */
int rme_picture_build_planes(void* ctx, int32_t pic_id, void* stream);

/* Copy one search plane of an uploaded reference to the host: plane 0 is
 * the padded integer plane, H.264 planes 1..3 are b, h, j (Hpel::plane
 * 0..2), HEVC planes 1..15 the fractional phase fy*4+fx (HalfPlanes'
 * planes[phase-1]). `rows` and `cols` receive the padded geometry
 * (height + 2*pad, width + 2*pad; H.264 at the coded size); `out` (may be
 * NULL) receives rows*cols samples. Synchronous. */
int rme_picture_download_plane(void* ctx, int32_t pic_id, int32_t plane, void* out,
                               int32_t* rows, int32_t* cols);

/* Bytes of device memory held by the context's pictures. */
int rme_memory_used(void* ctx, uint64_t* bytes);

/* ---- search --------------------------------------------------------------- */

/* Number of results rme_frame_search writes for `f` under `p`: njobs in
 * GIVEN mode; in STANDALONE mode one per (block, reference) for HEVC in
 * the order of rme_standalone_blocks, one per macroblock for H.264. */
int rme_frame_result_count(void* ctx, const rme_frame* f, const rme_params* p,
                           int32_t* count);

/* The STANDALONE blocks of a frame, in result order (HEVC: size levels from
 * the largest, raster order within a level, then the AMP units hevc_amp
 * asks for: per level of 16 or more, per CU in raster order, per mode in
 * bit order, the top/left unit then the other; H.264: macroblock raster).
 * `blocks` receives 4 int32 per block (x, y, w, h); pass NULL to get the
 * count only. */
int rme_standalone_blocks(const rme_picture_desc* d, const rme_params* p,
                          int32_t* blocks, int32_t* count);

/* Search one frame. Results go to `out` (host memory, count from
 * rme_frame_result_count). Synchronous: returns when `out` is written. */
int rme_frame_search(void* ctx, const rme_frame* f, const rme_params* p,
                     rme_result* out, void* stream);

/* Search many frames in one persistent launch: frames[i] with params[i];
 * results of frame i at out + offsets[i] (offsets from prefix sums of
 * rme_frame_result_count). The launch pulls (block, reference) tasks from
 * one device work queue that interleaves all frames, and is replayed as a
 * CUDA graph when the same batch shape comes again. */
int rme_batch_search(void* ctx, const rme_frame* frames, const rme_params* params,
                     int32_t nframes, rme_result* out, const int64_t* offsets,
                     void* stream);

/* The asynchronous forms of rme_frame_search / rme_batch_search (the
 * `rme_search(..., stream)` + `rme_sync` pair of the batched boundary): the
 * launch is queued on `stream` (NULL: the context's own) and the call
 * returns at once; `out` must be device memory or pinned host memory
 * (RME_EINVAL otherwise), and holds the results once the stream has reached
 * the end of the launch. This is what lets an encoder overlap its mode
 * decision for picture t (pick_pu, encode/h265_me.rs:1349,1363; p_mb,
 * encode/h264_analyse.rs:1957-1966) with the search of picture t+1. The
 * pictures the frames name must stay uploaded until rme_sync. At most four
 * launches of one context are in flight: a fifth call waits for the oldest
 * first (its error, if any, is kept for its stream's rme_sync). */
int rme_frame_search_async(void* ctx, const rme_frame* f, const rme_params* p,
                           rme_result* out, void* stream);
int rme_batch_search_async(void* ctx, const rme_frame* frames, const rme_params* params,
                           int32_t nframes, rme_result* out, const int64_t* offsets,
                           void* stream);

/* Wait for every asynchronous search of this context queued on `stream`
 * (NULL: the context's own) and report how they went: 0 when all were
 * complete and correct; RME_EDEVICE with `device_status` (may be NULL) set
 * to the device status bits when a kernel reported a failure (1: a bounded
 * wait ran out, 2: a malformed task); the first other error otherwise.
 * rme_last_stats then describes the last launch finished. */
int rme_sync(void* ctx, void* stream, uint32_t* device_status);

/* The STANDALONE decision over a frame's HEVC results (host side, cheap):
 * per block the reference with the least cost + lambda * ref_idx bits, and
 * the quadtree of 2Nx2N sizes whose summed costs are least. `best` gets one
 * int32 per block (chosen reference, -1 where no reference was searched);
 * `part` gets, per 8x8 cell of the picture, log2 of the chosen PU size. */
int rme_hevc_decide(const rme_picture_desc* d, const rme_params* p, int32_t nref,
                    const rme_result* res, int32_t* best, uint8_t* part);

/* Statistics of the last search call on this context. */
int rme_last_stats(void* ctx, rme_stats* s);

/* ---- weighted prediction (explicit weights) ----------------------------- */

/* A weighted reference's search plane: resident picture `dst_id` becomes
 * `ref_id`'s padded luma with the explicit weighting applied to every
 * sample, border included, clipped to the sample range, and its search
 * planes are built from it. H.264 weighted_search_plane
 * (h264_me.rs:653-672): ((v * weight + 2^(log_wd-1)) >> log_wd) + offset,
 * no rounding at log_wd 0 — the plane PRef::search / BRefs::search the
 * whole-sample search and its refinement score against. HEVC
 * weighted_search_plane (h265_me.rs:4275-4293): (((v << (14 - bd)) *
 * weight + 2^(log_wd-1)) >> log_wd) + offset, log_wd >= 1 — the plane the
 * whole-sample search of a weighted list scores against (the reference
 * refines sub-sample vectors on the unweighted reference under weighted
 * scoring, which this library does not reproduce). `offset` is at the
 * sample depth. Use `dst_id` as any other reference. Asynchronous on
 * `stream`. */
int rme_picture_weighted(void* ctx, int32_t ref_id, int32_t dst_id, int32_t log_wd, int32_t weight,
                         int32_t offset, void* stream);

/* The weight fit's moments of picture `cur_id` against `ref_id` over the
 * picture (wp_moments, dsp/distortion.rs:206-226): out[0..4] = sums of r,
 * c, r*r, r*c and |c - r|. Synchronous. */
int rme_wp_moments(void* ctx, int32_t cur_id, int32_t ref_id, uint64_t* out, void* stream);

/* weighted_sad (dsp/distortion.rs:228-252) over the picture: the sum of
 * |clip(((r * weight + 2^(shift-1)) >> shift) + offset) - c| (no rounding
 * at shift 0), `offset` at the sample depth. Synchronous. */
int rme_weighted_sad(void* ctx, int32_t cur_id, int32_t ref_id, int32_t weight, int32_t shift, int32_t offset,
                     uint64_t* out, void* stream);

/* ---- B pictures: bi-prediction (HEVC) ---------------------------------- */

/* A B unit's two one-list searches are GIVEN jobs of rme_frame_search whose
 * `ref` indexes a reference list holding both lists' pictures (pick_pu_b,
 * h265_me.rs:1768-1840, runs search_full + refine_subpel per list and
 * reference exactly as pick_pu does). What B adds is scored here: the bi
 * trial of a vector pair and its refinement, batched.
 *
 * One bi-prediction job: a block, the reference each list predicts from
 * (indexes into the frame's ref_ids), the pair's vectors, and for
 * rme_bi_refine the list searched again with that list's AMVP pair. */
typedef struct {
  int32_t x, y;        /* block position in luma samples                   */
  int32_t w, h;        /* block size, multiples of 4, at most 64           */
  int32_t ref[2];      /* list 0's and list 1's reference                  */
  rme_mv  mv[2];       /* the pair's quarter-sample vectors                */
  int32_t list;        /* rme_bi_refine: the list searched again (0, 1)    */
  rme_mv  mvp[2];      /* rme_bi_refine: that list's AMVP predictors       */
} rme_bi_job;

/* satd_bi_at (h265_me.rs:4209-4264) under default weighting, per job: the
 * SATD of the source block against the pair's bi-prediction. Where both
 * vectors' blocks can be read (a whole-sample vector within the plane's
 * border, a fractional one within HalfPlanes' reach on a phase HalfPlanes
 * builds: all fifteen up to 2,200,000 luma samples, the three half phases
 * above), the two one-list predictions averaged, (a + b + 1) >> 1;
 * elsewhere the exact bi-prediction of the 14-bit intermediates at
 * 15 - bit_depth. `f` names the source and the references (jobs unused);
 * `p` gives hevc_pad. Host jobs and output, synchronous. */
int rme_bi_satd(void* ctx, const rme_frame* f, const rme_params* p, const rme_bi_job* jobs, int32_t n,
                uint32_t* satd, void* stream);

/* satd_bi_at's explicit-weighting arm (h265_me.rs:4247-4261) per job: both
 * lists' 14-bit predictions (predict14, whatever the vectors) combined by
 * weighted_bi (dsp/hevc.rs:1064-1086),
 *   clip(((a * w0 + b * w1 + ((o0 + o1 + 1) << log2_wd)) >> (log2_wd + 1)),
 * and the SATD of the source block against it. log2_wd 0..14, weights
 * -128..255, offsets (at the sample depth) within +-4096; otherwise as
 * rme_bi_satd. Host jobs and output, synchronous. */
int rme_bi_satd_weighted(void* ctx, const rme_frame* f, const rme_params* p, const rme_bi_job* jobs, int32_t n,
                         int32_t log2_wd, int32_t w0, int32_t w1, int32_t o0, int32_t o1, uint32_t* satd,
                         void* stream);

/* refine_bi (h265_me.rs:3933-4014) per job: the other list's prediction
 * held fixed, list `list` searched again against the target
 * clip(2 * src - other's prediction) — search_full from the list's
 * current vector, then refine_subpel — at twice the SATD Lagrangian, with
 * the job's AMVP pair. One result per job (mv is the vector refine_bi
 * returns; cost and satd are against the target). Host jobs and output,
 * synchronous. */
int rme_bi_refine(void* ctx, const rme_frame* f, const rme_params* p, const rme_bi_job* jobs, int32_t n,
                  rme_result* out, void* stream);

/* A weighted list's sub-sample refinement (HEVC): refine_subpel
 * (h265_me.rs:3868-3922) with every candidate scored by satd_at_weighted's
 * explicit arm (4057-4073) — the reference's 14-bit prediction through
 * weighted_uni (dsp/hevc.rs:1036-1062) at log2_wd, weight and offset (the
 * list's luma weighting, offset at the sample depth) — on the unweighted
 * reference, as pick_pu does for a weighted list after its whole-sample
 * search on the weighted plane (rme_picture_weighted). `f` holds GIVEN jobs:
 * each job's seeds[0] is the whole-sample start, mvp its AMVP pair. One
 * result per job (int_mv the start). Host jobs and output, synchronous. */
int rme_hevc_weighted_refine(void* ctx, const rme_frame* f, const rme_params* p, int32_t log2_wd,
                             int32_t weight, int32_t offset, rme_result* out, void* stream);

/* ---- B macroblocks: the joint bi refinement (H.264) --------------------- */

/* One pair to refine jointly: a block of a B macroblock, each list's
 * reference (indexes into the frame's ref_ids), the pair's start vectors
 * and each list's rate predictor, and `limit`: a pair whose start already
 * costs more is left as it is (b_mb's bi_ratio gate; UINT32_MAX refines
 * every pair). */
typedef struct {
  int32_t x, y;        /* block position in luma samples                   */
  int32_t w, h;        /* 4, 8 or 16 each                                  */
  int32_t ref[2];      /* list 0's and list 1's reference                  */
  rme_mv  mv[2];       /* start vectors, quarter samples                   */
  rme_mv  mvp[2];      /* each list's predictor (MvCostTable::of)          */
  uint32_t limit;
} rme_h264_bi_job;

/* b_mb's bi_refine (h264_analyse.rs:2793-2900) per job, default weighting:
 * cost = SATD of the two lists' quarter-sample predictions averaged,
 * (p0 + p1 + 1) >> 1, plus both vectors' MvCostTable rates at the params'
 * QP; then up to `rounds` rounds, each list in turn: the ring of 8 points
 * (4 with `diamond`: bi_refine / bi_diamond) around that list's vector, the
 * other held, taken in order where strictly cheaper (a point whose rate
 * alone reaches the best is skipped), until a round moves nothing. Out:
 * the pair (mv_out, 2 per job) and its cost. Every vector a job can reach
 * (start +- rounds quarter samples) must lie inside search_bounds of its
 * reference (the planes the reference scores from; RME_EINVAL otherwise).
 * Host jobs and outputs, synchronous. */
int rme_h264_bi_refine(void* ctx, const rme_frame* f, const rme_params* p, const rme_h264_bi_job* jobs,
                       int32_t n, int32_t rounds, int32_t diamond, rme_mv* mv_out, uint32_t* cost_out,
                       void* stream);

/* ---- chroma of chosen vectors -------------------------------------------- */

/* Chroma prediction of chosen luma vectors (4:2:0): HEVC predict_block's
 * chroma arm (hevc/inter.rs:555-660, 4-tap EPEL_FILTERS, eighth samples,
 * uni rounding) or H.264 chroma_pred_into (h264_me.rs:812-837, bilinear).
 * blocks: 4 int32 per block (luma x, y, w, h); mvs: one per block.
 * out: per block (w/2)*(h/2) Cb samples then as many Cr, blocks packed in
 * order, sample type of the picture. */
int rme_chroma_predict(void* ctx, int32_t ref_id, int32_t nblocks,
                       const int32_t* blocks, const rme_mv* mvs, void* out,
                       void* stream);

/* ---- DSP kernels, batched (dsp/distortion.rs SadFn / SatdFn) -------------- */

/* Device-pointer batch of the reference's size-generic distortion kernels:
 * for i < n, out[i] = sad|satd(a + a_off[i], a_stride, b + b_off[i],
 * b_stride, w, h) over samples of `bit_depth` (uint8_t at 8, else uint16_t).
 * All pointers are device pointers; asynchronous on `stream`. */
int rme_sad_batch(const void* a, int64_t a_stride, const int64_t* a_off,
                  const void* b, int64_t b_stride, const int64_t* b_off,
                  int32_t w, int32_t h, int32_t bit_depth, int32_t n,
                  uint32_t* out, void* stream);
int rme_satd_batch(const void* a, int64_t a_stride, const int64_t* a_off,
                   const void* b, int64_t b_stride, const int64_t* b_off,
                   int32_t w, int32_t h, int32_t bit_depth, int32_t n,
                   uint32_t* out, void* stream);

/* ---- serving loop --------------------------------------------------------- */

/* A request loop on one context (a C++ host thread that owns it). Streams
 * are admitted against an HBM budget; each stream keeps its reference
 * pictures resident. Requests are per-frame ME calls; each starts on the
 * device as it arrives, beside the work already there (`mode`: a launch of
 * its own on one of three launch streams, or the resident search kernel's
 * queue).
 * open_stream, submit, poll and close_stream may be called from any host
 * threads at once; stop once, after the others have returned. While a
 * server runs, its context takes no other calls. The first frame of a
 * stream has no reference and is not searched (`out` may be NULL for it;
 * its completion reports 0 results). */
typedef struct {
  uint64_t hbm_budget_bytes;  /* admission limit for resident pictures      */
  int32_t  max_frames_per_launch;
  int32_t  max_streams;
  int32_t  mode;              /* RME_SERVE_LAUNCHES or RME_SERVE_RESIDENT     */
  int32_t  reserved;          /* 0                                           */
} rme_serve_opts;

/* Serving modes. LAUNCHES (0): the frames that arrived since the last launch
 * go into one search launch of their own as soon as one of three launch
 * streams is free, so up to three launches overlap on the device (a launch
 * of one or two frames runs the latency form). RESIDENT (1): one search
 * kernel stays on the GPU and frames join its queue as they arrive. */
#define RME_SERVE_LAUNCHES 0
#define RME_SERVE_RESIDENT 1

typedef struct {
  int64_t  request_id;
  int32_t  stream_id;
  int32_t  status;            /* 0 ok, else RME_E*                           */
  double   submit_s;          /* host clock (s) at submit                    */
  double   done_s;            /* host clock (s) when results were complete  */
  int32_t  nresults;
} rme_completion;

int rme_serve_start(void* ctx, const rme_serve_opts* o, void** server);
/* Admit a stream of one format and settings (STANDALONE predictors, 1..4
 * references); refused with RME_EBUSY when its resident pictures would pass
 * the budget. A stream holds nref + 4 pictures: up to four of its frames
 * join one launch. */
int rme_serve_open_stream(void* server, int32_t stream_id, const rme_picture_desc* d,
                          const rme_params* p, int32_t nref);
/* Submit one frame of a stream: its luma (host memory, copied before
 * return). The frame is searched against the stream's resident references
 * and then becomes its newest reference. Results land in `out` (host
 * memory the caller keeps until the completion is seen). */
int rme_serve_submit(void* server, int32_t stream_id, const void* luma,
                     rme_result* out, int64_t* request_id);
/* Completed requests since the last call (non-blocking). */
int rme_serve_poll(void* server, rme_completion* done, int32_t max, int32_t* n);
int rme_serve_close_stream(void* server, int32_t stream_id);
int rme_serve_stop(void* server);

/* ---- lookahead at half resolution ------------------------------------------- */

/* Both encoders' lookaheads (quantiser propagation) measure at half
 * resolution, in 8x8 blocks (16x16 of the picture), one set of kernels per
 * codec chosen by the picture's codec:
 *  - HEVC (encode/h265_cutree.rs): the picture reduced to 8 bits as 2x2
 *    means over ceil(w/2) x ceil(h/2), whole blocks;
 *  - H.264 (encode/h264_lookahead.rs): 2x2 means at the stream's sample
 *    depth, one block per macroblock.
 * Both planes are padded by 24 replicated samples. Batched per picture. */

/* Build (or rebuild) a resident picture's half-resolution plane and its
 * blocks' intra costs: HEVC LowRes::new + intra_cost (h265_cutree.rs:61-140,
 * the least SATD of DC, H and V floored at 16); H.264 Lookahead::add +
 * intra_costs (h264_lookahead.rs:87-222, the least SATD of DC, V, H and the
 * edge blend, plus 12). Synchronous. */
int rme_lowres_build(void* ctx, int32_t pic_id, void* stream);

/* Its block grid and (when `intra` is not NULL) the intra cost per block,
 * raster order. */
int rme_lowres_info(void* ctx, int32_t pic_id, int32_t* bw, int32_t* bh, uint32_t* intra);

/* The block search of every block of `cur_id` against `ref_id` (both built
 * with rme_lowres_build, same codec and size), the left and above blocks'
 * vectors as candidates:
 *  - HEVC search (h265_cutree.rs:152-216): seeds zero, left, above; a cross
 *    descent at steps 4, 2, 1 within +-16 of the best seed;
 *    SAD + 2 * min(|dx| + |dy|, 32);
 *  - H.264 search (h264_lookahead.rs:227-376): zero, then left and above
 *    clamped to the window (16 samples into the border, 32 at most);
 *    hexagon steps (at most 16), then the eight-point square;
 *    SAD + 2 * min(|dx| + |dy|, 64).
 * Per block the winner's SATD (`cost`), its vector in half-resolution
 * samples, and (when `nsad` is not NULL) the SADs the reference scores.
 * Host outputs, synchronous. */
int rme_lowres_search(void* ctx, int32_t cur_id, int32_t ref_id, uint32_t* cost, rme_mv* mv, uint32_t* nsad,
                      void* stream);

/* rme_lowres_search over `npairs` (cur_ids[k], ref_ids[k]) pairs in one
 * launch — a lookahead's estimates of many pictures at once (its depth of
 * pictures, each against the references it costs). All pictures share one
 * format. Outputs pair after pair (npairs x blocks each). Host outputs,
 * synchronous. */
int rme_lowres_search_batch(void* ctx, int32_t npairs, const int32_t* cur_ids, const int32_t* ref_ids,
                            uint32_t* cost, rme_mv* mv, uint32_t* nsad, void* stream);

/* The average-of-two cost of every block (HEVC bi_cost,
 * h265_cutree.rs:222-243; H.264 estimate, h264_lookahead.rs:417-432): the
 * SATD against the rounded average of its blocks displaced by mv0 in r0 and
 * mv1 in r1. Host inputs and output, synchronous. */
int rme_lowres_bi_cost(void* ctx, int32_t cur_id, int32_t r0_id, const rme_mv* mv0, int32_t r1_id,
                       const rme_mv* mv1, uint32_t* cost, void* stream);

/* ---- search without allocating --------------------------------------------- */

/* One picture's planes in device memory the caller owns, in the layout the
 * library keeps them (rme_picture_download_plane returns the same samples):
 * `nplanes` consecutive planes `plane_elems` samples apart, each padded by
 * `pad` samples on every side and `stride` samples per row; plane 0 is the
 * integer plane, then H.264's b, h, j or HEVC's fractional phases 1..15.
 * `base` (16-byte aligned) points at row 0, column 0 of plane 0, and the
 * memory must extend 16 bytes past the last plane. */
typedef struct {
  const void* base;
  int64_t plane_elems;
  int32_t stride;
  int32_t pad;
} rme_plane_set;

/* No counterpart in the reference (its search runs on the CPU and borrows
 * slices). A GIVEN-mode search that allocates no device memory, for callers
 * that cannot call cudaMalloc: a plugin whose host pipeline owns all of the
 * GPU's memory, or a latency-bound loop that cannot afford the device-wide
 * synchronisation of an allocation. Inputs and outputs are the caller's:
 * `src` (plane 0 read) and `refs[nref]` (all planes read) as above, `jobs`
 * and `out` (njobs each) in device memory. The same results as
 * rme_frame_search in GIVEN mode. The search's scratch lives in a fixed
 * device array of 541,952 bytes (about 529 KiB) inside the library, held on
 * every device it is used on until the process exits: at most 65536 jobs per
 * call (RME_EINVAL beyond). Parameters are held to the same limits as every
 * other search (RME_EINVAL). The jobs are in device memory, so the host
 * cannot check them: the kernel checks each job (reference index, seed
 * count, block size and position) before it reads anything the job names,
 * skips a job that fails and the call returns RME_EDEVICE; the other jobs'
 * results are written as usual. The first call on a device looks the array
 * up (do it before any stream capture); calls share the array, so calls
 * that overlap on the GPU race and must be serialised. The call returns
 * once the search on `stream` has finished (it synchronises the stream). */
int rme_search_given_noalloc(const rme_picture_desc* d, const rme_params* p, const rme_plane_set* src,
                             const rme_plane_set* refs, int32_t nref, const rme_job* jobs, int32_t njobs,
                             rme_result* out, void* stream);

/* ---- diagnostics ------------------------------------------------------------ */

/* Measured 32-bit integer-ALU throughput of `device` (add/shift/xor chains
 * over every SM), in operations per second: the roofline denominator of the
 * search kernel, which is integer work with no tensor-core content. */
int rme_probe_int_peak(int32_t device, double* ops_per_s);

/* The failure path of the library's bounded device waits (no counterpart
 * in the reference, whose ME does not wait on a device): one wait of the
 * lookahead's wavefront on a flag that nothing sets, limited to `polls`
 * polls (1..2^22, with back-off up to 256 ns each). It gives up, `status`
 * gets the timeout bit the searches report as RME_EDEVICE (1), and the
 * device stays usable; `seconds` (may be NULL) is how long the wait took. */
int rme_probe_wait_timeout(int32_t device, uint32_t polls, uint32_t* status, double* seconds);

#ifdef __cplusplus
}
#endif
#endif /* RIVET_ME_H */
