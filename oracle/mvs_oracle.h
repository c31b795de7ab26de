/*
 * mvs_oracle.h — CPU oracle for the dense-MVS path (TEST INFRASTRUCTURE).
 *
 * A restatement of the reference `mvs` crate in C++ (mvs/src/stereo.rs,
 * mvs/src/fuse.rs, the host glue of mvs/src/lib.rs, and Cam/Pose of
 * sfm-lite/src/geom.rs).  Only the tests, the smoke check and bench.py's CPU
 * baseline use it, as the checker; the product library never links it.
 *
 * PARITY UNPINNED: the reference is Rust, no Rust toolchain exists where this
 * was built, and the reference ships no tests or golden vectors.  The oracle
 * is pinned only by hand-derived known answers and by an independent
 * pure-Python restatement on small inputs (tests/golden/).
 */
#ifndef MVS_ORACLE_H
#define MVS_ORACLE_H

#include <stdint.h>
#include "../include/rcmvs.h"

#ifdef __cplusplus
extern "C" {
#endif

void orc_census_map(const uint8_t* gray, int32_t w, int32_t h, uint64_t* out);

uint64_t orc_pixel_rng(int32_t x, int32_t y, uint64_t salt);
uint64_t orc_next_u64(uint64_t* s);
float orc_uniform(uint64_t* s);
float orc_gauss(uint64_t* s);
int32_t orc_f32_to_i32(float v);

void orc_cam_normalize(double f, double cx, double cy, double k, double u, double v,
                       double* out2);

/* Rays of RefWorkspace::new (f64 normalize cast to f32). */
void orc_rays(const rcmvs_view* v, float* rx, float* ry);
/* rs = R_s R_r^T, ts = t_s - rs t_r (f64, cast to f32). */
void orc_rel_pose(const rcmvs_view* ref, const rcmvs_view* src, float* rs9, float* ts3);

/* plane_cost at every pixel for a given field (see rcmvs_plane_cost_field). */
int orc_plane_cost_field(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                         const int32_t* srcs, int32_t n_src, const float* planes,
                         const float* hints, float* cost_out, int32_t* hsum_out,
                         int32_t nthreads);

/* stereo::estimate_depth.  normal_out nullable.  nthreads<=0: all cores.
 * work_out (nullable) receives {cost evaluations, 5-term rows}. */
int orc_estimate_depth(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                       const int32_t* srcs, int32_t n_src, double zmin, double zmax,
                       const rcmvs_options* opts, float* depth_out, float* cost_out,
                       float* normal_out, int32_t nthreads, uint64_t* work_out);

/* estimate_depth with the learned init (no reference counterpart): the plane
 * sweep of stereo.rs:247-269 is replaced, for pixels whose quarter cell
 * proposes a usable plane, by the best of n_local planes around it, as the
 * library's rcmvs_scene_estimate_depth_seeded computes it.  pred holds the
 * reference view's (w/4)*(h/4) cells of 16 f32 (t, normal xyz, confidence
 * logit, 11 unused).  seeded_out (nullable) gets the number of seeded pixels.
 * RCMVS_FLAG_INIT_ONLY in opts->flags leaves the passes out (both here and
 * in orc_estimate_depth). */
int orc_estimate_depth_seeded(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                              const int32_t* srcs, int32_t n_src, double zmin, double zmax,
                              const rcmvs_options* opts, const float* pred, float conf_thr,
                              int32_t n_local, float span, float* depth_out, float* cost_out,
                              float* normal_out, int32_t nthreads, uint64_t* seeded_out);
/* ln(c / (1 - c)) in f64 rounded to f32; -inf for c <= 0, +inf for c >= 1. */
float orc_logit_threshold(float conf_thr);

/* fuse::fuse_depth_maps.  Output sorted by voxel key (x, then y, then z).
 * *xyz_out / *rgb_out are malloc'ed; release with orc_free. */
int orc_fuse_depth_maps(const rcmvs_view* views, int32_t n_views,
                        const float* const* depth_maps, const int32_t* order_offsets,
                        const int32_t* order, const double* sparse_xyz, uint64_t n_sparse,
                        const rcmvs_options* opts, double** xyz_out, uint8_t** rgb_out,
                        uint64_t* n_out, uint64_t* n_candidates_out, int32_t nthreads);
/* The two halves of orc_fuse_depth_maps.  Candidates (fuse.rs:96-167) of the
 * views with a depth map and ref_mask[v] != 0 (all when ref_mask is NULL), in
 * view-then-pixel order; per_view (nullable) gets each view's count. */
int orc_fuse_candidates(const rcmvs_view* views, int32_t n_views, const float* const* depth_maps,
                        const int32_t* order_offsets, const int32_t* order, const uint8_t* ref_mask,
                        const rcmvs_options* opts, double** xyz_out, uint8_t** rgb_out, uint64_t* n_out,
                        uint64_t* per_view, int32_t nthreads);
/* Voxel dedup (fuse.rs:72-92, 176-214) of candidates in accumulation order. */
int orc_fuse_reduce(const double* xyz, const uint8_t* rgb, uint64_t n, const double* sparse_xyz, uint64_t n_sparse,
                    const rcmvs_options* opts, double** xyz_out, uint8_t** rgb_out, uint64_t* n_out);
void orc_free(void* p);

/* extract_sift (sfm-lite/src/sift.rs:435-555) on an image at working
 * resolution (gray w*h, rgb w*h*3): keypoints (x, y) n*2, descriptors
 * n*128, colours n*3 (malloc'ed; orc_free); n_raw (nullable) gets the
 * number of scale-space extrema kept by the fit and rejection tests. */
/* match_pair (sfm-lite/src/matching.rs:22-95) of two descriptor sets
 * (na x 128, nb x 128); out_a / out_b need min(na, nb) entries. */
void orc_match_pair(const float* a, uint32_t na, const float* b, uint32_t nb, double ratio, uint32_t* out_a,
                    uint32_t* out_b, uint64_t* n_out);
int orc_extract_sift(const uint8_t* gray, const uint8_t* rgb, int32_t w, int32_t h, uint32_t max_features,
                     double contrast_thr, double** pts_out, float** desc_out, uint8_t** colors_out,
                     uint64_t* n_out, uint64_t* n_raw_out);

int orc_write_ply_binary(const char* path, const double* xyz, const uint8_t* rgb,
                         uint64_t n);

/* save_depth_vis (mvs/src/fuse.rs:241-268): the grey image and lo/hi. */
void orc_depth_vis(const float* depth, int32_t w, int32_t h, uint8_t* out, float* lo_hi);

/* load_views' image preparation (mvs/src/lib.rs:183-194): `image` 0.24
 * resize_exact with the Triangle filter when (mw, mh) != (w, h), then
 * to_luma8 / to_rgb8.  channels 1-4 (alpha dropped); gray mw*mh, rgb mw*mh*3. */
void orc_resize_view(const uint8_t* img, int32_t w, int32_t h, int32_t channels, int32_t mw, int32_t mh,
                     uint8_t* gray, uint8_t* rgb);

/* Host glue of run_mvs; same output layout as rcmvs_plan.  has_depth
 * (nullable) marks views that have a depth map; NULL means "every view with
 * at least one source". */
int orc_plan(const rcmvs_sparse* sparse, const rcmvs_view* views, int32_t n_views,
             const rcmvs_options* opts, int32_t* src_offsets, int32_t* srcs,
             double* zrange, int32_t* fuse_offsets, int32_t* fuse_order);

#ifdef __cplusplus
}
#endif
#endif
