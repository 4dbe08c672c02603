//! FFI declarations of librivet_me.so for the rivet-h26x crate
//! (`src/encode/me_cuda/sys.rs` in the crate): every entry point and struct
//! of `include/rivet_me.h`, field for field and parameter for parameter.
//! The header is the authority; this module mirrors it for a Rust caller.
#![allow(non_camel_case_types)]
use std::os::raw::{c_char, c_void};

#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_mv { pub x: i16, pub y: i16 }
#[repr(C)] pub struct rme_picture_desc { pub codec: i32, pub bit_depth: i32, pub width: i32, pub height: i32, pub stride: i32 }
#[repr(C)] #[derive(Clone, Copy)] pub struct rme_params {
    pub codec: i32, pub qp: i32, pub predictor_mode: i32,
    pub h264_range: i32, pub h264_hpel_iters: i32, pub h264_qpel_iters: i32,
    pub h264_umh: i32, pub h264_qpel_diamond: i32, pub h264_dia: i32,
    pub h264_refine_ratio: f32, pub h264_vertical_range: i32, pub h264_pad: i32,
    pub hevc_search_range: i32, pub hevc_search_rings: i32, pub hevc_quarter_cross: i32,
    pub hevc_lambda_scale: f32, pub hevc_pad: i32, pub hevc_pu_mask: i32, pub hevc_amp: i32,
}
#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_job {
    pub x: i32, pub y: i32, pub w: i32, pub h: i32, pub r#ref: i32, pub nseeds: i32, pub flags: i32,
    pub mvp: [rme_mv; 2], pub seeds: [rme_mv; 10],
}
#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_result {
    pub mv: rme_mv, pub r#ref: i32, pub cost: u32, pub satd: u32,
    pub int_mv: rme_mv, pub int_cost: u32, pub n_sad: u32, pub n_satd: u32,
}
#[repr(C)] pub struct rme_frame {
    pub src_id: i32, pub nref: i32, pub ref_ids: [i32; 4], pub jobs: *const rme_job, pub njobs: i32,
}
#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_h264_bi_job {
    pub x: i32, pub y: i32, pub w: i32, pub h: i32, pub r#ref: [i32; 2], pub mv: [rme_mv; 2],
    pub mvp: [rme_mv; 2], pub limit: u32,
}
#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_bi_job {
    pub x: i32, pub y: i32, pub w: i32, pub h: i32, pub r#ref: [i32; 2], pub mv: [rme_mv; 2],
    pub list: i32, pub mvp: [rme_mv; 2],
}
#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_stats {
    pub tasks: u64, pub sad_candidates: u64, pub satd_candidates: u64,
    pub sad_samples: u64, pub satd_samples: u64, pub kernel_ms: f32, pub planes_ms: f32,
}
#[repr(C)] #[derive(Clone, Copy)] pub struct rme_plane_set {
    pub base: *const c_void, pub plane_elems: i64, pub stride: i32, pub pad: i32,
}
#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_serve_opts {
    pub hbm_budget_bytes: u64, pub max_frames_per_launch: i32, pub max_streams: i32, pub mode: i32,
    pub reserved: i32,
}
#[repr(C)] #[derive(Clone, Copy, Default)] pub struct rme_completion {
    pub request_id: i64, pub stream_id: i32, pub status: i32, pub submit_s: f64, pub done_s: f64,
    pub nresults: i32,
}

extern "C" {
    pub fn rme_params_default(p: *mut rme_params, codec: i32, qp: i32);
    pub fn rme_ctx_create(ctx: *mut *mut c_void, device: i32) -> i32;
    pub fn rme_ctx_destroy(ctx: *mut c_void);
    pub fn rme_last_error(ctx: *mut c_void) -> *const c_char;
    pub fn rme_picture_upload(ctx: *mut c_void, pic_id: i32, d: *const rme_picture_desc,
                              luma: *const c_void, as_ref: i32, stream: *mut c_void) -> i32;
    pub fn rme_picture_release(ctx: *mut c_void, pic_id: i32) -> i32;
    pub fn rme_frame_search(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params,
                            out: *mut rme_result, stream: *mut c_void) -> i32;
    pub fn rme_batch_search(ctx: *mut c_void, frames: *const rme_frame, params: *const rme_params,
                            n: i32, out: *mut rme_result, offsets: *const i64, stream: *mut c_void) -> i32;
    pub fn rme_frame_search_async(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params,
                                  out: *mut rme_result, stream: *mut c_void) -> i32;
    pub fn rme_batch_search_async(ctx: *mut c_void, frames: *const rme_frame, params: *const rme_params,
                                  n: i32, out: *mut rme_result, offsets: *const i64, stream: *mut c_void) -> i32;
    pub fn rme_sync(ctx: *mut c_void, stream: *mut c_void, device_status: *mut u32) -> i32;
    pub fn rme_picture_upload_chroma(ctx: *mut c_void, pic_id: i32, cb: *const c_void, cr: *const c_void,
                                     cstride: i32, stream: *mut c_void) -> i32;
    pub fn rme_chroma_predict(ctx: *mut c_void, ref_id: i32, nblocks: i32, blocks: *const i32,
                              mvs: *const rme_mv, out: *mut c_void, stream: *mut c_void) -> i32;
    pub fn rme_sad_batch(a: *const c_void, a_stride: i64, a_off: *const i64, b: *const c_void, b_stride: i64,
                         b_off: *const i64, w: i32, h: i32, bit_depth: i32, n: i32, out: *mut u32,
                         stream: *mut c_void) -> i32;
    pub fn rme_satd_batch(a: *const c_void, a_stride: i64, a_off: *const i64, b: *const c_void, b_stride: i64,
                          b_off: *const i64, w: i32, h: i32, bit_depth: i32, n: i32, out: *mut u32,
                          stream: *mut c_void) -> i32;
    pub fn rme_lowres_build(ctx: *mut c_void, pic_id: i32, stream: *mut c_void) -> i32;
    pub fn rme_lowres_info(ctx: *mut c_void, pic_id: i32, bw: *mut i32, bh: *mut i32, intra: *mut u32) -> i32;
    pub fn rme_lowres_search(ctx: *mut c_void, cur_id: i32, ref_id: i32, cost: *mut u32, mv: *mut rme_mv,
                             nsad: *mut u32, stream: *mut c_void) -> i32;
    pub fn rme_lowres_search_batch(ctx: *mut c_void, npairs: i32, cur_ids: *const i32, ref_ids: *const i32,
                                   cost: *mut u32, mv: *mut rme_mv, nsad: *mut u32, stream: *mut c_void) -> i32;
    pub fn rme_lowres_bi_cost(ctx: *mut c_void, cur_id: i32, r0_id: i32, mv0: *const rme_mv, r1_id: i32,
                              mv1: *const rme_mv, cost: *mut u32, stream: *mut c_void) -> i32;
    pub fn rme_picture_weighted(ctx: *mut c_void, ref_id: i32, dst_id: i32, log_wd: i32, weight: i32,
                                offset: i32, stream: *mut c_void) -> i32;
    pub fn rme_wp_moments(ctx: *mut c_void, cur_id: i32, ref_id: i32, out: *mut u64, stream: *mut c_void) -> i32;
    pub fn rme_weighted_sad(ctx: *mut c_void, cur_id: i32, ref_id: i32, weight: i32, shift: i32, offset: i32,
                            out: *mut u64, stream: *mut c_void) -> i32;
    pub fn rme_hevc_weighted_refine(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params, log2_wd: i32,
                                    weight: i32, offset: i32, out: *mut rme_result, stream: *mut c_void) -> i32;
    pub fn rme_h264_bi_refine(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params,
                              jobs: *const rme_h264_bi_job, n: i32, rounds: i32, diamond: i32,
                              mv_out: *mut rme_mv, cost_out: *mut u32, stream: *mut c_void) -> i32;
    pub fn rme_bi_satd(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params, jobs: *const rme_bi_job,
                       n: i32, satd: *mut u32, stream: *mut c_void) -> i32;
    pub fn rme_bi_satd_weighted(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params,
                                jobs: *const rme_bi_job, n: i32, log2_wd: i32, w0: i32, w1: i32, o0: i32, o1: i32,
                                satd: *mut u32, stream: *mut c_void) -> i32;
    pub fn rme_bi_refine(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params, jobs: *const rme_bi_job,
                         n: i32, out: *mut rme_result, stream: *mut c_void) -> i32;
    pub fn rme_picture_build_planes(ctx: *mut c_void, pic_id: i32, stream: *mut c_void) -> i32;
    pub fn rme_picture_download_plane(ctx: *mut c_void, pic_id: i32, plane: i32, out: *mut c_void,
                                      rows: *mut i32, cols: *mut i32) -> i32;
    pub fn rme_memory_used(ctx: *mut c_void, bytes: *mut u64) -> i32;
    pub fn rme_frame_result_count(ctx: *mut c_void, f: *const rme_frame, p: *const rme_params,
                                  count: *mut i32) -> i32;
    pub fn rme_standalone_blocks(d: *const rme_picture_desc, p: *const rme_params, blocks: *mut i32,
                                 count: *mut i32) -> i32;
    pub fn rme_hevc_decide(d: *const rme_picture_desc, p: *const rme_params, nref: i32, res: *const rme_result,
                           best: *mut i32, part: *mut u8) -> i32;
    pub fn rme_last_stats(ctx: *mut c_void, s: *mut rme_stats) -> i32;
    pub fn rme_search_given_noalloc(d: *const rme_picture_desc, p: *const rme_params, src: *const rme_plane_set,
                                    refs: *const rme_plane_set, nref: i32, jobs: *const rme_job, njobs: i32,
                                    out: *mut rme_result, stream: *mut c_void) -> i32;
    pub fn rme_serve_start(ctx: *mut c_void, o: *const rme_serve_opts, server: *mut *mut c_void) -> i32;
    pub fn rme_serve_open_stream(server: *mut c_void, stream_id: i32, d: *const rme_picture_desc,
                                 p: *const rme_params, nref: i32) -> i32;
    pub fn rme_serve_submit(server: *mut c_void, stream_id: i32, luma: *const c_void, out: *mut rme_result,
                            request_id: *mut i64) -> i32;
    pub fn rme_serve_poll(server: *mut c_void, done: *mut rme_completion, max: i32, n: *mut i32) -> i32;
    pub fn rme_serve_close_stream(server: *mut c_void, stream_id: i32) -> i32;
    pub fn rme_serve_stop(server: *mut c_void) -> i32;
    pub fn rme_probe_int_peak(device: i32, ops_per_s: *mut f64) -> i32;
    pub fn rme_probe_wait_timeout(device: i32, polls: u32, status: *mut u32, seconds: *mut f64) -> i32;
}
