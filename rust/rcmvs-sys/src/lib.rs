//! Raw bindings to librcmvs: the B200 (sm_100a) dense multi-view-stereo path
//! of RustCOLMAP's `mvs` crate (census patch-match stereo and
//! geometric-consistency fusion) behind the C ABI of `include/rcmvs.h`.
//!
//! Every declaration mirrors the header one for one; the header is the
//! authority on semantics (status codes, buffer ownership, limits).  The
//! reference functions these stand in for, as paths within RustCOLMAP:
//!
//! | reference | here |
//! |---|---|
//! | `stereo::estimate_depth` (`mvs/src/stereo.rs:234-241`) | [`rcmvs_estimate_depth`], batched [`rcmvs_estimate_depth_batch`] |
//! | `fuse::fuse_depth_maps` (`mvs/src/fuse.rs:64-71`) | [`rcmvs_fuse_depth_maps`] |
//! | `fuse::write_ply_binary` (`mvs/src/fuse.rs:222`) | [`rcmvs_write_ply_binary`] |
//! | `run_mvs` (`mvs/src/lib.rs:294-300`) | [`rcmvs_run_mvs`] + the caller's image decoding and file output |
//! | `MvsOptions` (`mvs/src/lib.rs:33-54`) | [`rcmvs_options`] |
//! | `ViewData` (`mvs/src/lib.rs:86-101`) | [`rcmvs_view`] (grey as u8 luma) |
//!
//! The crate links `librcmvs.so` from `RCMVS_LIB_DIR` (see `build.rs`).
#![allow(non_camel_case_types, non_snake_case)]

use std::os::raw::{c_char, c_int, c_void};

pub const RCMVS_OK: c_int = 0;
pub const RCMVS_E_ARG: c_int = -1;
pub const RCMVS_E_CUDA: c_int = -2;
pub const RCMVS_E_NOMEM: c_int = -3;
pub const RCMVS_E_LIMIT: c_int = -4;
pub const RCMVS_E_IO: c_int = -5;
pub const RCMVS_E_STATE: c_int = -6;

pub const RCMVS_MAX_SOURCES: u32 = 32;

pub const RCMVS_FLAG_ONE_CANDIDATE: u32 = 1;
pub const RCMVS_FLAG_PERSISTENT: u32 = 2;
pub const RCMVS_FLAG_CUDA_GRAPH: u32 = 4;
pub const RCMVS_FLAG_AUTOTUNE: u32 = 8;
pub const RCMVS_FLAG_NO_SKIP_DUPLICATES: u32 = 16;
pub const RCMVS_FLAG_INIT_ONLY: u32 = 32;
pub const RCMVS_FLAG_SEED_AND_SWEEP: u32 = 64;
pub const RCMVS_FLAG_ROW_STEP_INIT: u32 = 128;
pub const RCMVS_FLAG_NO_REPEAT_SKIP: u32 = 256;
pub const RCMVS_FLAG_LOCKSTEP_PASSES: u32 = 512;
pub const RCMVS_MAX_PASSES: u32 = 4096;

pub const RCMVS_NOALLOC_MAX_PIXELS: u32 = 307200;
pub const RCMVS_NOALLOC_MAX_SOURCES: u32 = 4;
pub const RCMVS_NOALLOC_SCRATCH_BYTES: u64 = 38416384;

/// `mvs::MvsOptions` field for field, then the extensions.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rcmvs_options {
    pub max_dim: u32,
    pub num_sources: u32,
    pub sweeps: u32,
    pub num_hyp: u32,
    pub min_consistent: u32,
    pub save_depth_vis: u32,
    pub cost_thr: f32,
    pub passes: u32,
    pub depth_diff: f64,
    pub voxel_rel: f64,
    pub reproj_px: f64,
    pub tile_w: u32,
    pub tile_h: u32,
    pub flags: u32,
    pub threads_per_pixel: u32,
}

/// One registered view at working resolution (`mvs::ViewData`).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct rcmvs_view {
    pub w: i32,
    pub h: i32,
    pub f: f64,
    pub cx: f64,
    pub cy: f64,
    pub k: f64,
    pub R: [f64; 9],
    pub t: [f64; 3],
    pub gray: *const u8,
    pub rgb: *const u8,
}

/// The arguments of one `stereo::estimate_depth` call.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct rcmvs_job {
    pub ref_idx: i32,
    pub n_src: i32,
    pub srcs: *const i32,
    pub zmin: f64,
    pub zmax: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct rcmvs_depth_out {
    pub depth: *mut f32,
    pub cost: *mut f32,
    pub normal: *mut f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct rcmvs_sparse {
    pub n_points: u64,
    pub xyz: *const f64,
    pub track_offsets: *const u64,
    pub track_views: *const i32,
}

/// Library-allocated cloud; release with [`rcmvs_points_free`].
#[repr(C)]
#[derive(Debug)]
pub struct rcmvs_points {
    pub n: u64,
    pub xyz: *mut f64,
    pub rgb: *mut u8,
}

/// `mvs::MvsStats` plus timings.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rcmvs_stats {
    pub views: u64,
    pub views_with_depth: u64,
    pub dense_points: u64,
    pub fusion_candidates: u64,
    pub elapsed_s: f32,
    pub stereo_s: f32,
    pub fuse_s: f32,
    pub reserved0: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rcmvs_tune_entry {
    pub w: i32,
    pub h: i32,
    pub tile_w: i32,
    pub tile_h: i32,
    pub threads_per_pixel: i32,
    pub reserved: i32,
    pub ms_best: f32,
    pub ms_default: f32,
}

/// `sift::SiftOptions`.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rcmvs_sift_options {
    pub max_dim: u32,
    pub max_features: u32,
    pub reserved: u32,
    pub reserved2: u32,
    pub contrast_thr: f64,
}

/// `sift::SiftFrame` without the name; release with [`rcmvs_sift_frame_free`].
#[repr(C)]
#[derive(Debug)]
pub struct rcmvs_sift_frame {
    pub width: i32,
    pub height: i32,
    pub n: u64,
    pub n_raw: u64,
    pub pts: *mut f64,
    pub desc: *mut f32,
    pub colors: *mut u8,
}

/// Matches of a batch of pairs; release with [`rcmvs_matches_free`].
#[repr(C)]
#[derive(Debug)]
pub struct rcmvs_matches {
    pub n_pairs: u64,
    pub offsets: *mut u64,
    pub a: *mut u32,
    pub b: *mut u32,
}

/// Opaque handles.
#[repr(C)]
pub struct rcmvs_ctx {
    _private: [u8; 0],
}
#[repr(C)]
pub struct rcmvs_scene {
    _private: [u8; 0],
}
#[repr(C)]
pub struct rcmvs_net {
    _private: [u8; 0],
}

extern "C" {
    /// MvsOptions::default() (mvs/src/lib.rs:56-70); extensions off.
pub fn rcmvs_options_default(opts: *mut rcmvs_options);
    pub fn rcmvs_pass_count(opts: *const rcmvs_options) -> u64;
    /// Releases a library-allocated cloud.
    pub fn rcmvs_points_free(pts: *mut rcmvs_points);
    /// A context on CUDA device `device` (with its own stream).
    pub fn rcmvs_ctx_create(device: c_int, out: *mut *mut rcmvs_ctx) -> c_int;
    pub fn rcmvs_ctx_destroy(ctx: *mut rcmvs_ctx);
    pub fn rcmvs_last_error(ctx: *const rcmvs_ctx) -> *const c_char;
    pub fn rcmvs_ctx_stream(ctx: *mut rcmvs_ctx) -> *mut c_void;
    pub fn rcmvs_ctx_synchronize(ctx: *mut rcmvs_ctx) -> c_int;
    pub fn rcmvs_diag_wait_timeout(ctx: *mut rcmvs_ctx, limit_ns: u64) -> c_int;
    pub fn rcmvs_version() -> *const c_char;
    /// census_map (mvs/src/lib.rs:119-142).  Host buffers.
    pub fn rcmvs_census(ctx: *mut rcmvs_ctx, gray: *const u8, w: i32, h: i32, census_out: *mut u64) -> c_int;
    /// Working size of load_views (mvs/src/lib.rs:155-157, 185-187).
    pub fn rcmvs_working_size(w: i32, h: i32, max_dim: u32, mw: *mut i32, mh: *mut i32) -> c_int;
    /// load_views' Triangle resize + to_luma8/to_rgb8 (mvs/src/lib.rs:183-194).
    pub fn rcmvs_resize_view(ctx: *mut rcmvs_ctx, img: *const u8, w: i32, h: i32, channels: i32, mw: i32, mh: i32,
                             gray_out: *mut u8, rgb_out: *mut u8) -> c_int;
    /// stereo::estimate_depth (mvs/src/stereo.rs:234-394).  Host buffers.
    pub fn rcmvs_estimate_depth(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32, ref_idx: i32,
                                srcs: *const i32, n_src: i32, zmin: f64, zmax: f64, opts: *const rcmvs_options,
                                depth_out: *mut f32, cost_out: *mut f32, normal_out: *mut f32) -> c_int;
    /// The rayon loop over views calling estimate_depth (mvs/src/lib.rs:351-374), one batch.
    pub fn rcmvs_estimate_depth_batch(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32,
                                      jobs: *const rcmvs_job, n_jobs: i32, opts: *const rcmvs_options,
                                      outs: *const rcmvs_depth_out) -> c_int;
    /// fuse::fuse_depth_maps (mvs/src/fuse.rs:64-215).
    pub fn rcmvs_fuse_depth_maps(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32,
                                 depth_maps: *const *const f32, order_offsets: *const i32, order: *const i32,
                                 sparse_xyz: *const f64, n_sparse: u64, opts: *const rcmvs_options,
                                 out: *mut rcmvs_points) -> c_int;
    /// The consistency half of fuse_depth_maps (mvs/src/fuse.rs:96-167) for a subset of reference views.
    pub fn rcmvs_fuse_candidates(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32,
                                 depth_maps: *const *const f32, order_offsets: *const i32, order: *const i32,
                                 ref_views: *const i32, n_ref: i32, opts: *const rcmvs_options,
                                 out: *mut rcmvs_points, per_view: *mut u64) -> c_int;
    /// The voxel-dedup half of fuse_depth_maps (mvs/src/fuse.rs:72-92, 176-214).
    pub fn rcmvs_fuse_reduce(ctx: *mut rcmvs_ctx, xyz: *const f64, rgb: *const u8, n: u64, sparse_xyz: *const f64,
                             n_sparse: u64, opts: *const rcmvs_options, out: *mut rcmvs_points) -> c_int;
    /// fuse::write_ply_binary (mvs/src/fuse.rs:222-239), byte-identical.
    pub fn rcmvs_write_ply_binary(path: *const c_char, xyz: *const f64, rgb: *const u8, n: u64) -> c_int;
    /// The files run_mvs writes into <out>/dense (mvs/src/lib.rs:429-501).
    pub fn rcmvs_write_dense_outputs(dense_dir: *const c_char, xyz: *const f64, rgb: *const u8, n: u64,
                                     stats: *const rcmvs_stats, web_cap: u64) -> c_int;
    /// run_mvs host glue: covisibility, sources, depth ranges, fusion order (mvs/src/lib.rs:224-282, 303-342, 398-418).
    pub fn rcmvs_plan(sparse: *const rcmvs_sparse, views: *const rcmvs_view, n_views: i32,
                      opts: *const rcmvs_options, src_offsets: *mut i32, srcs: *mut i32, zrange: *mut f64,
                      fuse_offsets: *mut i32, fuse_order: *mut i32) -> c_int;
    /// The dense stage of run_mvs (mvs/src/lib.rs:294-517) without image decoding or file output.
    pub fn rcmvs_run_mvs(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32, sparse: *const rcmvs_sparse,
                         opts: *const rcmvs_options, depth_outs: *const rcmvs_depth_out, out: *mut rcmvs_points,
                         stats: *mut rcmvs_stats) -> c_int;
    pub fn rcmvs_scene_create(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32,
                              out: *mut *mut rcmvs_scene) -> c_int;
    pub fn rcmvs_scene_destroy(scene: *mut rcmvs_scene);
    pub fn rcmvs_scene_prepare(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene) -> c_int;
    pub fn rcmvs_scene_estimate_depth(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, jobs: *const rcmvs_job,
                                      n_jobs: i32, opts: *const rcmvs_options) -> c_int;
    pub fn rcmvs_autotune(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, jobs: *const rcmvs_job, n_jobs: i32,
                          opts: *const rcmvs_options) -> c_int;
    pub fn rcmvs_tune_table(ctx: *mut rcmvs_ctx, out: *mut rcmvs_tune_entry, cap: i32, n_out: *mut i32) -> c_int;
    pub fn rcmvs_tune_set(ctx: *mut rcmvs_ctx, entries: *const rcmvs_tune_entry, n: i32) -> c_int;
    pub fn rcmvs_scene_fuse(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, order_offsets: *const i32,
                            order: *const i32, sparse_xyz: *const f64, n_sparse: u64, opts: *const rcmvs_options,
                            n_points_out: *mut u64) -> c_int;
    pub fn rcmvs_scene_fuse_candidates(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, order_offsets: *const i32,
                                       order: *const i32, ref_views: *const i32, n_ref: i32,
                                       opts: *const rcmvs_options, out: *mut rcmvs_points, per_view: *mut u64) -> c_int;
    pub fn rcmvs_scene_get_depth(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, view: i32, depth: *mut f32,
                                 cost: *mut f32, normal: *mut f32) -> c_int;
    /// Device-to-device moves of depth maps and fusion candidates (one scene over several processes).
    pub fn rcmvs_scene_depth_to_device(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, view: i32, depth_dev: *mut f32) -> c_int;
    pub fn rcmvs_scene_set_depth(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, view: i32, depth: *const f32,
                                 on_device: i32) -> c_int;
    pub fn rcmvs_scene_fuse_candidates_device(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene,
                                              order_offsets: *const i32, order: *const i32, ref_views: *const i32,
                                              n_ref: i32, opts: *const rcmvs_options, n_out: *mut u64,
                                              per_view: *mut u64) -> c_int;
    pub fn rcmvs_scene_candidates_to_device(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, xyz_dev: *mut f64,
                                            rgb_dev: *mut u8) -> c_int;
    pub fn rcmvs_scene_fuse_reduce_device(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, xyz_dev: *const f64,
                                          rgb_dev: *const u8, n: u64, sparse_xyz: *const f64, n_sparse: u64,
                                          opts: *const rcmvs_options, n_points_out: *mut u64) -> c_int;
    pub fn rcmvs_scene_get_census(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, view: i32, census: *mut u64) -> c_int;
    pub fn rcmvs_scene_get_points(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, xyz: *mut f64, rgb: *mut u8,
                                  ply_body: *mut u8) -> c_int;
    /// fuse::save_depth_vis (mvs/src/fuse.rs:241-268): the grey image.
    pub fn rcmvs_depth_vis(ctx: *mut rcmvs_ctx, depth: *const f32, w: i32, h: i32, out: *mut u8, lo_hi: *mut f32) -> c_int;
    pub fn rcmvs_scene_depth_vis(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, view: i32, out: *mut u8,
                                 lo_hi: *mut f32) -> c_int;
    pub fn rcmvs_write_png_gray(path: *const c_char, img: *const u8, w: i32, h: i32) -> c_int;
    /// SiftOptions::default() (sfm-lite/src/sift.rs:27-31).
    pub fn rcmvs_sift_options_default(opts: *mut rcmvs_sift_options);
    /// sift::extract_sift (sfm-lite/src/sift.rs:435-555).
    pub fn rcmvs_extract_sift(ctx: *mut rcmvs_ctx, img: *const u8, w: i32, h: i32, channels: i32,
                              opts: *const rcmvs_sift_options, out: *mut rcmvs_sift_frame) -> c_int;
    pub fn rcmvs_sift_frame_free(frame: *mut rcmvs_sift_frame);
    /// matching::match_pair (sfm-lite/src/matching.rs:22-95) for a batch of pairs.
    pub fn rcmvs_match_pairs(ctx: *mut rcmvs_ctx, desc: *const *const f32, n_desc: *const i32, n_frames: i32,
                             pairs: *const i32, n_pairs: i32, ratio: f64, out: *mut rcmvs_matches) -> c_int;
    pub fn rcmvs_matches_free(matches: *mut rcmvs_matches);
    /// plane_cost (mvs/src/stereo.rs:158-228) at every pixel for a given plane field (diagnostic).
    pub fn rcmvs_plane_cost_field(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32, ref_idx: i32,
                                  srcs: *const i32, n_src: i32, planes: *const f32, hints: *const f32,
                                  cost_out: *mut f32, hsum_out: *mut i32) -> c_int;
    pub fn rcmvs_last_work(ctx: *mut rcmvs_ctx, cost_evals: *mut u64, rows: *mut u64) -> c_int;
    pub fn rcmvs_ctx_timing(ctx: *mut rcmvs_ctx, enable: c_int) -> c_int;
    pub fn rcmvs_ctx_kernel_time(ctx: *mut rcmvs_ctx, name: *const c_char, ms_total: *mut f64, launches: *mut u64) -> c_int;
    pub fn rcmvs_selftest_f2i(ctx: *mut rcmvs_ctx, in_: *const f32, n: i32, out: *mut i32) -> c_int;
    pub fn rcmvs_net_param_count() -> u64;
    pub fn rcmvs_net_create(ctx: *mut rcmvs_ctx, params: *const f32, seed: u64, out: *mut *mut rcmvs_net) -> c_int;
    pub fn rcmvs_net_destroy(net: *mut rcmvs_net);
    pub fn rcmvs_net_get_params(net: *mut rcmvs_net, out: *mut f32) -> c_int;
    pub fn rcmvs_net_forward(ctx: *mut rcmvs_ctx, net: *mut rcmvs_net, x_dev: *const c_void, n: i32, h: i32, w: i32,
                             out_dev: *mut f32) -> c_int;
    pub fn rcmvs_net_train_step(ctx: *mut rcmvs_ctx, net: *mut rcmvs_net, x_dev: *const c_void,
                                labels_dev: *const f32, n: i32, h: i32, w: i32, lr: f32, apply: i32,
                                loss_out: *mut f32, grads_host: *mut f32) -> c_int;
    pub fn rcmvs_scene_costvol(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, jobs: *const rcmvs_job, n_jobs: i32,
                               out_dev: *mut c_void) -> c_int;
    /// Stereo seeded by the proposal network (no reference counterpart).
    pub fn rcmvs_scene_estimate_depth_learned(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, jobs: *const rcmvs_job,
                                              n_jobs: i32, opts: *const rcmvs_options, net: *mut rcmvs_net,
                                              conf_thr: f32, n_local: i32, span: f32, learned_pixels: *mut u64) -> c_int;
    /// Stereo seeded by caller-given proposals (no reference counterpart).
    pub fn rcmvs_scene_estimate_depth_seeded(ctx: *mut rcmvs_ctx, scene: *mut rcmvs_scene, jobs: *const rcmvs_job,
                                             n_jobs: i32, opts: *const rcmvs_options, pred: *const f32,
                                             pred_on_device: i32, conf_thr: f32, n_local: i32, span: f32,
                                             learned_pixels: *mut u64) -> c_int;
    /// rcmvs_run_mvs with stereo seeded by the network (no reference counterpart).
    pub fn rcmvs_run_mvs_learned(ctx: *mut rcmvs_ctx, views: *const rcmvs_view, n_views: i32,
                                 sparse: *const rcmvs_sparse, opts: *const rcmvs_options, net: *mut rcmvs_net,
                                 conf_thr: f32, n_local: i32, span: f32, depth_outs: *const rcmvs_depth_out,
                                 out: *mut rcmvs_points, stats: *mut rcmvs_stats) -> c_int;
    /// estimate_depth for callers that cannot allocate device memory (no reference counterpart).
    pub fn rcmvs_estimate_depth_noalloc(views: *const rcmvs_view, n_views: i32, ref_idx: i32, srcs: *const i32,
                                        n_src: i32, zmin: f64, zmax: f64, opts: *const rcmvs_options,
                                        depth_dev: *mut f32, cost_dev: *mut f32, stream: *mut c_void) -> c_int;
}

/// A context that destroys itself, and the one error type of the binding.
pub mod safe {
    use super::*;
    use std::ffi::CStr;

    #[derive(Debug)]
    pub struct Error {
        pub code: c_int,
        pub message: String,
    }

    pub struct Context {
        ptr: *mut rcmvs_ctx,
    }

    impl Context {
        /// A context on CUDA device `device`.
        pub fn new(device: c_int) -> Result<Context, Error> {
            let mut p: *mut rcmvs_ctx = std::ptr::null_mut();
            let rc = unsafe { rcmvs_ctx_create(device, &mut p) };
            if rc != RCMVS_OK {
                return Err(Error { code: rc, message: format!("no context on CUDA device {device}") });
            }
            Ok(Context { ptr: p })
        }

        pub fn as_ptr(&self) -> *mut rcmvs_ctx {
            self.ptr
        }

        /// Turns a status into a Result with the context's last message.
        pub fn check(&self, rc: c_int) -> Result<(), Error> {
            if rc == RCMVS_OK {
                return Ok(());
            }
            let msg = unsafe { CStr::from_ptr(rcmvs_last_error(self.ptr)) }.to_string_lossy().into_owned();
            Err(Error { code: rc, message: msg })
        }
    }

    impl Drop for Context {
        fn drop(&mut self) {
            unsafe { rcmvs_ctx_destroy(self.ptr) }
        }
    }

    /// `MvsOptions::default()` with the extensions off.
    pub fn default_options() -> rcmvs_options {
        let mut o = rcmvs_options::default();
        unsafe { rcmvs_options_default(&mut o) };
        o
    }
}
