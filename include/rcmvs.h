/*
 * rcmvs.h — C ABI of the B200-native dense multi-view-stereo path.
 *
 * This library replaces the `mvs` crate of RustCOLMAP (census patch-match
 * stereo + geometric-consistency fusion).  Every entry point below names the
 * reference function it stands in for (paths are relative to the reference
 * project root).  The ABI is plain C: POD structs, raw pointers, sizes and an
 * int status.  No CUDA or torch type appears in a signature.
 *
 * Conventions
 *  - Status: RCMVS_OK (0) on success, a negative RCMVS_E_* code otherwise;
 *    rcmvs_last_error(ctx) then holds a one-line message.
 *  - Host buffers are caller-owned unless a function says it allocates
 *    (rcmvs_points, freed with rcmvs_points_free).
 *  - One rcmvs_ctx per device.  A context is not thread-safe; separate
 *    contexts are independent.  All device work of a context runs on its
 *    own CUDA stream (rcmvs_ctx_stream).
 *  - Views are supplied at the stereo working resolution: a view whose
 *    long side exceeds opts->max_dim is rejected.  The reference's resize to
 *    `max_dim` (mvs/src/lib.rs:185-192) is a separate call,
 *    rcmvs_resize_view, made while loading images.
 *  - Image rows are row-major, pixel (x, y) at index y*w + x.  A pixel's
 *    centre sits at integer coordinates (sfm-lite/src/geom.rs:28-42).
 */
#ifndef RCMVS_H
#define RCMVS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RCMVS_OK 0
#define RCMVS_E_ARG (-1)     /* invalid argument (null pointer, bad size, bad index) */
#define RCMVS_E_CUDA (-2)    /* a CUDA runtime call failed */
#define RCMVS_E_NOMEM (-3)   /* device or host allocation failed */
#define RCMVS_E_LIMIT (-4)   /* a documented size limit was exceeded */
#define RCMVS_E_IO (-5)      /* file output failed */
#define RCMVS_E_STATE (-6)   /* call order violated (e.g. fuse before depth) */

#define RCMVS_MAX_SOURCES 32 /* support views per reference view */

/* Mirrors `mvs::MvsOptions` (mvs/src/lib.rs:33-54) field for field; the
 * extension fields at the end have no counterpart there. */
typedef struct rcmvs_options {
    uint32_t max_dim;        /* longest image side used for stereo */
    uint32_t num_sources;    /* support views per reference view (K) */
    uint32_t sweeps;         /* patch-match sweeps; passes = 2*max(sweeps,1) */
    uint32_t num_hyp;        /* plane-sweep hypotheses; max(num_hyp,2) used */
    uint32_t min_consistent; /* min OTHER views agreeing in fusion */
    uint32_t save_depth_vis; /* PNGs are written by the callers that write files
                                (see rcmvs_depth_vis); rcmvs_run_mvs writes none */
    float cost_thr;          /* max census Hamming fraction of a valid pixel */
    uint32_t passes;         /* extension: Jacobi passes; 0 = 2*max(sweeps,1), the
                                reference's schedule (rcmvs_pass_count).  The
                                perturbation scales anneal over the passes run
                                (t = pass / passes), as over 2*sweeps.  At most
                                RCMVS_MAX_PASSES. */
    double depth_diff;       /* relative depth agreement in fusion */
    double voxel_rel;        /* voxel cell / robust sparse bbox diagonal */
    /* ---- extensions (no reference counterpart) ---- */
    double reproj_px;        /* >0: fusion also requires the forward-backward
                                reprojection error to be <= reproj_px pixels;
                                0 = off (reference behaviour) */
    uint32_t tile_w;         /* stereo tile width in pixels; 0 = default (8) */
    uint32_t tile_h;         /* stereo tile height in pixels; 0 = default (8) */
    uint32_t flags;          /* RCMVS_FLAG_* bits; 0 = defaults */
    uint32_t threads_per_pixel; /* Jacobi passes: 0 or 1 = one thread per pixel
                                (default: streamed, see
                                RCMVS_FLAG_LOCKSTEP_PASSES); 5 = five lanes per
                                pixel, one per window column (tiles of at most
                                128 pixels).  Same results bit for bit. */
} rcmvs_options;

/* The plane-sweep init evaluates each pixel's hypotheses one at a time, a
 * warp waiting at every hypothesis for its slowest lane, instead of the
 * default table sweep (RCMVS_FLAG_ROW_STEP_INIT).  Same results bit for
 * bit; kept for comparison.  The Jacobi passes are chosen by
 * threads_per_pixel and RCMVS_FLAG_LOCKSTEP_PASSES. */
#define RCMVS_FLAG_ONE_CANDIDATE 1u

/* Persistent (view, tile) work queue: each init/pass launch runs as many
 * blocks as stay resident on the GPU, and every block takes tile after tile
 * of the batch (all views, in job order) from an atomic counter instead of
 * computing the one tile of its block index.  Same results bit for bit. */
#define RCMVS_FLAG_PERSISTENT 2u

/* Capture the batch's launch schedule (init -> 2*max(sweeps,1) passes ->
 * gate) in a CUDA graph, cached on the scene and replayed while the job
 * table, options and buffers are unchanged.  Ignored while per-kernel
 * timing (rcmvs_ctx_timing) is on.  Same results bit for bit. */
#define RCMVS_FLAG_CUDA_GRAPH 4u

/* Per-resolution-class tile shapes from the autotuner (rcmvs_autotune):
 * classes not yet tuned on this context are tuned on the batch's jobs
 * first.  Overrides tile_w/tile_h.  Same results bit for bit. */
#define RCMVS_FLAG_AUTOTUNE 8u

/* Evaluate every candidate the way the reference does.  By default four
 * exact shortcuts run: a Jacobi pass skips a neighbour's plane that is bit
 * for bit the plane (normal and offset d) the pixel's stored cost was
 * computed with (its cost would be that same cost, or an early abort, and
 * never lower, so it can not be accepted); every evaluation (init and
 * passes) stops once its window sum reaches best_cost * 25K (the sum only
 * grows, so the candidate's cost could not be below the best and it could
 * not be kept); every evaluation also stops once the early-abort test
 * after the first row of the next support view is certain to fire (that
 * test divides by 5 * (view + 1), less than the current row's divisor, and
 * the sum only grows); and the repeat skip of RCMVS_FLAG_NO_REPEAT_SKIP.
 * None changes an output bit, only the work counters (rcmvs_last_work),
 * which with this flag count the reference's calls and rows. */
#define RCMVS_FLAG_NO_SKIP_DUPLICATES 16u

/* Diagnostic: run the init (plane sweep, or the learned init) and the gate
 * only, without the Jacobi passes, so the init's planes and costs can be
 * compared on their own.  Not a reference schedule. */
#define RCMVS_FLAG_INIT_ONLY 32u

/* Learned init only (rcmvs_scene_estimate_depth_learned / _seeded,
 * rcmvs_run_mvs_learned): a pixel seeded by a proposal also runs the
 * plane sweep, starting from the proposal's cost as its best so far (the
 * sweep's early-abort hint is then tight from the first hypothesis), and
 * keeps a sweep plane only when it is strictly cheaper.  Without it a seeded
 * pixel skips the sweep. */
#define RCMVS_FLAG_SEED_AND_SWEEP 64u

/* The plane sweep of the init by default walks the hypotheses block by
 * block: for each hypothesis and support view the window counts of a tile
 * and its halo are computed once into shared memory (on a fronto-parallel
 * plane a window cell's count does not depend on which pixel's window holds
 * it) and every pixel runs the reference's chain over them.  This flag
 * selects the row-step sweep instead (each lane streams its own hypotheses
 * one window row at a time).  Same results bit for bit. */
#define RCMVS_FLAG_ROW_STEP_INIT 128u

/* Turns off the repeat skip alone (it is also off under
 * RCMVS_FLAG_NO_SKIP_DUPLICATES).  By default a Jacobi pass does not
 * evaluate the plane of a neighbour that the previous pass left unchanged,
 * unless that pass refused the pixel's best candidate (n . ray <= 0.05):
 * the neighbour offered the same plane in the previous pass, where it could
 * not beat that pass's best, and whether a candidate beats a best value is
 * monotone in that value (a lower best only makes the early abort and the
 * rejection bound fire sooner), so it cannot win now.  The first pass after
 * the init evaluates every candidate.  Same results bit for bit; fewer
 * window rows. */
#define RCMVS_FLAG_NO_REPEAT_SKIP 256u

/* The Jacobi passes run one thread per pixel in lockstep (tiles of
 * tile_w x tile_h): a warp runs each candidate slot for as long as its
 * slowest lane needs.  By default (threads_per_pixel 0 or 1) a pass
 * streams the pixels of 16x16 tiles through blocks of 64 threads: each
 * lane evaluates its pixel's candidates one window row at a time, starts
 * the next candidate as soon as one ends and claims the tile's next pixel
 * as soon as its pixel ends.  The streamed passes run as persistent
 * launches and keep each block's random candidates in a device scratch of
 * the scene (48 bytes per tile pixel per resident block, about 29 MB on a
 * 148-SM GPU).  Same results bit for bit (and the same work counters);
 * tile_w/tile_h and the autotuner's shapes then apply to the init only. */
#define RCMVS_FLAG_LOCKSTEP_PASSES 512u

#define RCMVS_MAX_PASSES 4096u


/* Fills `MvsOptions::default()` (mvs/src/lib.rs:56-70); extensions off. */
void rcmvs_options_default(rcmvs_options* opts);
/* The Jacobi passes an estimate with `opts` runs: 0 with
 * RCMVS_FLAG_INIT_ONLY, else opts->passes when set, else
 * 2 * max(sweeps, 1) (mvs/src/stereo.rs:271). */
uint64_t rcmvs_pass_count(const rcmvs_options* opts);

/* One registered view at working resolution.  Replaces `mvs::ViewData`
 * (mvs/src/lib.rs:86-101) with the grey image as u8 (ViewData.gray is
 * u8/255 in f32, a strictly monotone map of the same values), the camera
 * as SIMPLE_RADIAL `Cam{f,cx,cy,k}` (sfm-lite/src/geom.rs:14-20) and the
 * world->camera pose `Pose{r,t}` (sfm-lite/src/geom.rs:50-54). */
typedef struct rcmvs_view {
    int32_t w, h;
    double f, cx, cy, k;
    double R[9];             /* row-major world->camera rotation */
    double t[3];
    const uint8_t* gray;     /* w*h luma */
    const uint8_t* rgb;      /* w*h*3 colour, may be NULL when not fusing */
} rcmvs_view;

/* One depth-estimation job: reference view + ordered support views and the
 * depth range.  The arguments of `stereo::estimate_depth`
 * (mvs/src/stereo.rs:234-241). */
typedef struct rcmvs_job {
    int32_t ref_idx;
    int32_t n_src;
    const int32_t* srcs;     /* n_src view indices, in priority order */
    double zmin, zmax;
} rcmvs_job;

/* Per-job host outputs (w*h floats each; normal is 3*w*h, nullable). */
typedef struct rcmvs_depth_out {
    float* depth;            /* DepthMap.depth: z in the reference camera, 0 = invalid */
    float* cost;             /* DepthMap.cost: census Hamming fraction of the kept plane */
    float* normal;           /* extension: unit plane normal per pixel (nullable) */
} rcmvs_depth_out;

/* Sparse reconstruction subset the dense stage reads (colmap-io Point3D,
 * colmap-io/src/lib.rs:91-103).  Track entries are view indices; entries
 * outside [0, n_views) are ignored, as the reference ignores image ids it
 * has no view for (mvs/src/lib.rs:227-231). */
typedef struct rcmvs_sparse {
    uint64_t n_points;
    const double* xyz;             /* 3*n_points */
    const uint64_t* track_offsets; /* n_points+1 */
    const int32_t* track_views;    /* track_offsets[n_points] entries */
} rcmvs_sparse;

/* Fused point cloud: the `Vec<(f64,f64,f64,[u8;3])>` of
 * `fuse::fuse_depth_maps` (mvs/src/fuse.rs:64-71).  Points come out sorted
 * by voxel key (the reference's HashMap order is unspecified).  Arrays are
 * allocated by the library; release with rcmvs_points_free. */
typedef struct rcmvs_points {
    uint64_t n;
    double* xyz;             /* 3*n */
    uint8_t* rgb;            /* 3*n */
} rcmvs_points;
void rcmvs_points_free(rcmvs_points* pts);

/* Run statistics: `mvs::MvsStats` (mvs/src/lib.rs:72-79) plus timings. */
typedef struct rcmvs_stats {
    uint64_t views;
    uint64_t views_with_depth;
    uint64_t dense_points;
    uint64_t fusion_candidates;
    float elapsed_s, stereo_s, fuse_s;
    uint32_t reserved0;
} rcmvs_stats;

typedef struct rcmvs_ctx rcmvs_ctx;

/* Context on CUDA device `device` (creates its stream). */
int rcmvs_ctx_create(int device, rcmvs_ctx** out);
void rcmvs_ctx_destroy(rcmvs_ctx* ctx);
const char* rcmvs_last_error(const rcmvs_ctx* ctx);
/* The context's cudaStream_t, as an opaque pointer (for event timing). */
void* rcmvs_ctx_stream(rcmvs_ctx* ctx);
/* Blocks until the context's stream has drained.  Also returns
 * RCMVS_E_CUDA (message in rcmvs_last_error) if a tensor-core kernel
 * queued since the last call gave up one of its bounded waits for its MMAs
 * (the kernel then freed its tensor memory and returned early). */
int rcmvs_ctx_synchronize(rcmvs_ctx* ctx);
/* Diagnostic of that path: one block waits, with a limit of `limit_ns`
 * (1 us .. 1 s), on an mbarrier nothing arrives on, as the tensor-core
 * kernels wait for their MMAs, and sets the same fault word when the limit
 * runs out; the next rcmvs_ctx_synchronize then reports it.  Queued on the
 * context's stream. */
int rcmvs_diag_wait_timeout(rcmvs_ctx* ctx, uint64_t limit_ns);
const char* rcmvs_version(void);

/* ---------------------------------------------------------------- host API */

/* 7x7 census transform, 48 bits in a u64, bit (dy+3)*7+(dx+3) set iff the
 * clamped neighbour is darker than the centre.  Replaces `census_map`
 * (mvs/src/lib.rs:119-142).  Host buffers. */
int rcmvs_census(rcmvs_ctx* ctx, const uint8_t* gray, int32_t w, int32_t h,
                 uint64_t* census_out);

/* Working resolution of a w x h camera (mvs/src/lib.rs:155-157, :185-187):
 * s = min(max_dim / max(w, h), 1) in f64, side = max(round(side * s), 16). */
int rcmvs_working_size(int32_t w, int32_t h, uint32_t max_dim, int32_t* mw, int32_t* mh);

/* One decoded 8-bit image brought to the working resolution the way
 * `load_views` does (mvs/src/lib.rs:183-194): when (mw, mh) != (w, h),
 * `resize_exact(mw, mh, FilterType::Triangle)` of the `image` crate 0.24
 * (a vertical pass into f32, then a horizontal pass rounded to u8, each
 * output sample a normalised triangle-weighted sum of its input samples);
 * then `to_luma8` and `to_rgb8`.  `img` holds h rows of w pixels of
 * `channels` bytes: 1 grey, 2 grey + alpha, 3 RGB, 4 RGBA (alpha is
 * dropped; the colour channels resize independently).  gray_out gets mw*mh
 * bytes, rgb_out mw*mh*3 (host buffers; either may be NULL).  Sides up to
 * 2^23; mw, mh >= 1. */
int rcmvs_resize_view(rcmvs_ctx* ctx, const uint8_t* img, int32_t w, int32_t h, int32_t channels,
                      int32_t mw, int32_t mh, uint8_t* gray_out, uint8_t* rgb_out);

/* Depth (+cost, optional normal) map of one reference view.  Replaces
 * `stereo::estimate_depth` (mvs/src/stereo.rs:234-394). Host buffers. */
int rcmvs_estimate_depth(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                         int32_t ref_idx, const int32_t* srcs, int32_t n_src,
                         double zmin, double zmax, const rcmvs_options* opts,
                         float* depth_out, float* cost_out, float* normal_out);

/* Many `estimate_depth` calls in one batched launch sequence (the rayon
 * loop over views at mvs/src/lib.rs:351-374).  outs[i] receives job i. */
int rcmvs_estimate_depth_batch(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                               const rcmvs_job* jobs, int32_t n_jobs,
                               const rcmvs_options* opts, const rcmvs_depth_out* outs);

/* Geometric-consistency fusion + voxel dedup.  Replaces
 * `fuse::fuse_depth_maps` (mvs/src/fuse.rs:64-215).  depth_maps[v] is a
 * w*h map of view v or NULL (the reference's `None`); fusion view lists are
 * CSR: view v checks order[order_offsets[v] .. order_offsets[v+1]]. */
int rcmvs_fuse_depth_maps(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                          const float* const* depth_maps,
                          const int32_t* order_offsets, const int32_t* order,
                          const double* sparse_xyz, uint64_t n_sparse,
                          const rcmvs_options* opts, rcmvs_points* out);

/* Fusion in two halves, for a scene whose reference views are spread over
 * several processes (no reference counterpart; in the reference both halves
 * run inside `fuse::fuse_depth_maps`).  rcmvs_fuse_candidates runs the
 * consistency check of fuse.rs:96-167 for the pixels of ref_views only
 * (n_ref entries; views without a depth map contribute nothing) against
 * every view's depth map, and returns their candidates, the averaged point
 * and the reference pixel's colour, in view-then-pixel order (`out`,
 * library-allocated; per_view, nullable, n_views entries, gets each view's
 * count).  rcmvs_fuse_reduce is the voxel dedup of fuse.rs:72-92, 176-214 over
 * candidates given in the reference's accumulation order (view, then pixel):
 * the candidates of all reference views, concatenated in view order, give
 * exactly the cloud of rcmvs_fuse_depth_maps. */
int rcmvs_fuse_candidates(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                          const float* const* depth_maps,
                          const int32_t* order_offsets, const int32_t* order,
                          const int32_t* ref_views, int32_t n_ref,
                          const rcmvs_options* opts, rcmvs_points* out, uint64_t* per_view);
int rcmvs_fuse_reduce(rcmvs_ctx* ctx, const double* xyz, const uint8_t* rgb, uint64_t n,
                      const double* sparse_xyz, uint64_t n_sparse,
                      const rcmvs_options* opts, rcmvs_points* out);

/* Binary little-endian PLY, byte-identical to `fuse::write_ply_binary`
 * (mvs/src/fuse.rs:222-239). */
int rcmvs_write_ply_binary(const char* path, const double* xyz, const uint8_t* rgb,
                           uint64_t n);


/* The files `run_mvs` writes into <out>/dense after fusion
 * (mvs/src/lib.rs:429-501): dense.ply (as rcmvs_write_ply_binary),
 * dense_web.json (the decimated copy for web viewers: points farther from
 * the centroid than the robust radius dropped, then every ceil(kept / cap)-th
 * point, 4 decimals; none for an empty cloud) and, when stats is non-NULL,
 * mvs_stats.json.  dense_dir must exist.  web_cap 0 = the reference's
 * 400000.  Host only. */
int rcmvs_write_dense_outputs(const char* dense_dir, const double* xyz, const uint8_t* rgb, uint64_t n,
                              const rcmvs_stats* stats, uint64_t web_cap);

/* Host glue of `run_mvs` (mvs/src/lib.rs:303-342, :358, :398-418):
 * co-visibility counts, top-K support views (count >= 10), per-view depth
 * range, fusion order (sources first).  Outputs (caller-allocated):
 *   src_offsets[n_views+1], srcs[n_views*num_sources]   (CSR)
 *   zrange[2*n_views]                                   (zmin, zmax)
 *   fuse_offsets[n_views+1], fuse_order[n_views*n_views] (CSR)
 * Views without sources get no depth map and are left out of every fusion
 * order, as in the reference. */
int rcmvs_plan(const rcmvs_sparse* sparse, const rcmvs_view* views, int32_t n_views,
               const rcmvs_options* opts, int32_t* src_offsets, int32_t* srcs,
               double* zrange, int32_t* fuse_offsets, int32_t* fuse_order);

/* The dense stage of `run_mvs` (mvs/src/lib.rs:294-517) without image
 * decoding and without writing files: plan, batched stereo for every view
 * with sources, fusion.  depth_outs (nullable, n_views entries) receive the
 * depth maps; views without sources get depth 0 / cost 1.  `out` receives
 * the fused cloud; stats (nullable) the run statistics.  The call is
 * synchronous: the views' buffers are read until it returns (their RGB is
 * uploaded on a second stream of the context, beside the stereo) and all
 * of the call's GPU work has finished when it returns. */
int rcmvs_run_mvs(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                  const rcmvs_sparse* sparse, const rcmvs_options* opts,
                  const rcmvs_depth_out* depth_outs, rcmvs_points* out,
                  rcmvs_stats* stats);

/* -------------------------------------------------- device-resident API */
/* A scene keeps every view's grey/colour image, census, rays, planes,
 * depth/cost/normal maps and the fused cloud in device memory, so repeated
 * stereo and fusion calls move no image data across PCIe. */
typedef struct rcmvs_scene rcmvs_scene;

/* Uploads the views and runs census + ray kernels (device). */
int rcmvs_scene_create(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                       rcmvs_scene** out);
void rcmvs_scene_destroy(rcmvs_scene* scene);
/* Recomputes census + rays of every view of the scene on the device (the
 * census_map of mvs/src/lib.rs:198 and the rays of mvs/src/stereo.rs:118-125;
 * rcmvs_scene_create already ran it once).  Asynchronous. */
int rcmvs_scene_prepare(rcmvs_ctx* ctx, rcmvs_scene* scene);
/* Device-resident batched stereo; results stay on the device. Asynchronous
 * on the context stream. */
int rcmvs_scene_estimate_depth(rcmvs_ctx* ctx, rcmvs_scene* scene, const rcmvs_job* jobs,
                               int32_t n_jobs, const rcmvs_options* opts);

/* Tile-shape autotuner (no reference counterpart).  Reference views are
 * grouped into resolution classes by (w, h).  For every class of the given
 * jobs that this context has not tuned yet, the plane-sweep init and one
 * pass (with opts, on the class's first jobs up to about 1 Mpx) are timed
 * with CUDA events for each candidate shape and scored as init +
 * 2*max(sweeps,1) passes.  Candidates: 8x8, 16x4, 4x16 (64 threads), 16x16,
 * 32x8, 8x32, 64x4 (256), 16x8, 8x16, 32x4 (128) and 8x4, 4x8, 16x2 (32, one
 * warp per block).  One thread count is kept for all classes of a context
 * (the one with the least summed best score at the first tuning), and each
 * class gets its best shape of that count.  The trial overwrites the jobs'
 * plane buffers, not their depth maps.  Synchronous. */
typedef struct rcmvs_tune_entry {
    int32_t w, h;            /* resolution class */
    int32_t tile_w, tile_h;  /* chosen shape */
    int32_t threads_per_pixel; /* of the passes: 1 or 5 */
    int32_t reserved;
    float ms_best;           /* trial score of the chosen shape (ms) */
    float ms_default;        /* trial score of the 8x8 default (ms) */
} rcmvs_tune_entry;
int rcmvs_autotune(rcmvs_ctx* ctx, rcmvs_scene* scene, const rcmvs_job* jobs, int32_t n_jobs,
                   const rcmvs_options* opts);
/* Copies up to cap tuned classes of the context; *n_out = classes stored. */
int rcmvs_tune_table(rcmvs_ctx* ctx, rcmvs_tune_entry* out, int32_t cap, int32_t* n_out);
/* Replaces the context's table (e.g. one saved from an earlier run); each
 * shape must have tile_w*tile_h <= 256 pixels, a multiple of 32.  Jobs of
 * classes whose shapes differ in pixel count may share a launch (its blocks
 * then have the largest count of threads).  Later tuning keeps the thread
 * count of entries[0]. */
int rcmvs_tune_set(rcmvs_ctx* ctx, const rcmvs_tune_entry* entries, int32_t n);
/* Device-resident fusion of the scene's depth maps (views that were the
 * reference of a job have a map).  *n_points_out gets the fused count
 * (this call synchronises once to size the output). */
int rcmvs_scene_fuse(rcmvs_ctx* ctx, rcmvs_scene* scene, const int32_t* order_offsets,
                     const int32_t* order, const double* sparse_xyz, uint64_t n_sparse,
                     const rcmvs_options* opts, uint64_t* n_points_out);
/* rcmvs_fuse_candidates on the scene's device-resident depth maps. */
int rcmvs_scene_fuse_candidates(rcmvs_ctx* ctx, rcmvs_scene* scene, const int32_t* order_offsets,
                                const int32_t* order, const int32_t* ref_views, int32_t n_ref,
                                const rcmvs_options* opts, rcmvs_points* out, uint64_t* per_view);
/* Copies one view's maps to host buffers (any pointer may be NULL). */
int rcmvs_scene_get_depth(rcmvs_ctx* ctx, rcmvs_scene* scene, int32_t view, float* depth,
                          float* cost, float* normal);
/* Device-to-device moves of depth maps and fusion candidates, for callers
 * that exchange them between GPUs themselves (one scene sharded over
 * several processes, each with its own context; no reference counterpart).
 * All are asynchronous on the context stream: synchronise it
 * (rcmvs_ctx_synchronize) before another stream reads what they wrote, and
 * make the writes of another stream visible before calling them.
 *   rcmvs_scene_depth_to_device: one view's depth map (w*h f32) into a
 *     caller device buffer (RCMVS_E_STATE if the view has none).
 *   rcmvs_scene_set_depth: a view's depth map from a caller buffer (device
 *     memory when on_device != 0, else host memory, copied before return);
 *     the view then counts as having a map for fusion.
 *   rcmvs_scene_fuse_candidates_device: rcmvs_scene_fuse_candidates with the
 *     candidates kept in the scene; *n_out gets their count (this call
 *     synchronises once to learn it), per_view (nullable) the count per view.
 *   rcmvs_scene_candidates_to_device: the kept candidates (3 f64 + 3 u8
 *     each, view-then-pixel order) into caller device buffers.
 *   rcmvs_scene_fuse_reduce_device: the voxel dedup of rcmvs_fuse_reduce over
 *     n device-resident candidates into the scene's fused cloud (read it with
 *     rcmvs_scene_get_points); *n_points_out gets the count. */
int rcmvs_scene_depth_to_device(rcmvs_ctx* ctx, rcmvs_scene* scene, int32_t view, float* depth_dev);
int rcmvs_scene_set_depth(rcmvs_ctx* ctx, rcmvs_scene* scene, int32_t view, const float* depth,
                          int32_t on_device);
int rcmvs_scene_fuse_candidates_device(rcmvs_ctx* ctx, rcmvs_scene* scene, const int32_t* order_offsets,
                                       const int32_t* order, const int32_t* ref_views, int32_t n_ref,
                                       const rcmvs_options* opts, uint64_t* n_out, uint64_t* per_view);
int rcmvs_scene_candidates_to_device(rcmvs_ctx* ctx, rcmvs_scene* scene, double* xyz_dev, uint8_t* rgb_dev);
int rcmvs_scene_fuse_reduce_device(rcmvs_ctx* ctx, rcmvs_scene* scene, const double* xyz_dev,
                                   const uint8_t* rgb_dev, uint64_t n, const double* sparse_xyz,
                                   uint64_t n_sparse, const rcmvs_options* opts, uint64_t* n_points_out);
/* Copies one view's census (w*h u64) to the host. */
int rcmvs_scene_get_census(rcmvs_ctx* ctx, rcmvs_scene* scene, int32_t view,
                           uint64_t* census);
/* Copies the fused cloud (n from rcmvs_scene_fuse) to host buffers; ply_body
 * (nullable, 15*n bytes) receives the PLY vertex records the device packed. */
int rcmvs_scene_get_points(rcmvs_ctx* ctx, rcmvs_scene* scene, double* xyz, uint8_t* rgb,
                           uint8_t* ply_body);

/* Depth-map visualisation of `fuse::save_depth_vis` (mvs/src/fuse.rs:241-268)
 * on the GPU: the 2nd/98th percentiles of the valid depths (z > 0;
 * `ds[(n*0.02) as usize]`, `ds[(n*0.98) as usize - 1]`, or 0 and 1 below 32
 * valid pixels) set the scale; out[i] = 0 for invalid depth, else
 * (255 * (1 - clamp((z - lo) / range, 0, 1))) as u8, near = bright.
 * depth and out are host buffers of w*h; lo_hi (nullable) gets lo and hi.
 * Synchronous. */
int rcmvs_depth_vis(rcmvs_ctx* ctx, const float* depth, int32_t w, int32_t h, uint8_t* out,
                    float* lo_hi);
/* The same for a scene view's device-resident depth map (RCMVS_E_STATE if
 * the view has none). */
int rcmvs_scene_depth_vis(rcmvs_ctx* ctx, rcmvs_scene* scene, int32_t view, uint8_t* out,
                          float* lo_hi);
/* 8-bit greyscale PNG of a w*h image (the file `save_depth_vis` writes;
 * zlib-compressed, so its bytes differ from the `image` crate's while the
 * decoded pixels are the same).  Host only. */
int rcmvs_write_png_gray(const char* path, const uint8_t* img, int32_t w, int32_t h);

/* ------------------------------------------------------------------ SIFT */
/* `sift::SiftOptions` (sfm-lite/src/sift.rs:20-32). */
typedef struct rcmvs_sift_options {
    uint32_t max_dim;        /* longest image side used for extraction */
    uint32_t max_features;   /* cap after the response sort */
    uint32_t reserved;
    uint32_t reserved2;
    double contrast_thr;     /* on DoG values in [0,1] intensity units */
} rcmvs_sift_options;
/* Fills `SiftOptions::default()` (sift.rs:27-31): 1600, 2048, 0.0067. */
void rcmvs_sift_options_default(rcmvs_sift_options* opts);

/* `sift::SiftFrame` (sfm-lite/src/sift.rs:34-41) without the name; arrays
 * are allocated by the library (rcmvs_sift_frame_free). */
typedef struct rcmvs_sift_frame {
    int32_t width, height;   /* working size the keypoints refer to */
    uint64_t n;              /* keypoints */
    uint64_t n_raw;          /* scale-space extrema that passed the fit (diagnostic) */
    double* pts;             /* n * 2: x, y */
    float* desc;             /* n * 128, L2-normalised */
    uint8_t* colors;         /* n * 3: RGB at the rounded position */
} rcmvs_sift_frame;

/* SIFT extraction of one decoded 8-bit image (h rows of w pixels of
 * `channels` bytes, 1-4; alpha dropped).  Replaces `sift::extract_sift`
 * (sfm-lite/src/sift.rs:435-555): Triangle resize when the long side
 * exceeds max_dim, Gaussian pyramid and DoG, extrema with the quadratic fit
 * and the contrast / curvature tests, orientations, 4x4x8 descriptors,
 * response-sorted and capped. */
int rcmvs_extract_sift(rcmvs_ctx* ctx, const uint8_t* img, int32_t w, int32_t h, int32_t channels,
                       const rcmvs_sift_options* opts, rcmvs_sift_frame* out);
void rcmvs_sift_frame_free(rcmvs_sift_frame* frame);

/* Matches of a batch of image pairs; pair p's matches are
 * a[offsets[p] .. offsets[p+1]) (indices into the first frame's keypoints,
 * ascending) and b[...] (into the second's).  Library-allocated
 * (rcmvs_matches_free). */
typedef struct rcmvs_matches {
    uint64_t n_pairs;
    uint64_t* offsets;       /* n_pairs + 1 */
    uint32_t* a;
    uint32_t* b;
} rcmvs_matches;

/* `matching::match_pair` (sfm-lite/src/matching.rs:22-95) for n_pairs pairs
 * (pairs[2p], pairs[2p+1]) of frames whose descriptors are desc[f]
 * (n_desc[f] x 128 floats each): mutual nearest neighbours by squared L2
 * distance, summed in f32 in the reference's order, with Lowe's ratio test
 * (`ratio`, cast to f32) both ways and the 0.9 absolute cap. */
int rcmvs_match_pairs(rcmvs_ctx* ctx, const float* const* desc, const int32_t* n_desc, int32_t n_frames,
                      const int32_t* pairs, int32_t n_pairs, double ratio, rcmvs_matches* out);
void rcmvs_matches_free(rcmvs_matches* matches);

/* ---------------------------------------------------------- diagnostics */

/* `plane_cost` (mvs/src/stereo.rs:158-228) evaluated at every pixel of the
 * reference view for a caller-given plane field: planes[4*i..] = (nx, ny,
 * nz, d) and hints[i] (early-abort hint; +inf disables).  cost_out[i] is
 * bit-identical to the reference (1e9 when aborted); hsum_out (nullable)
 * receives the integer Hamming sum of the evaluated in-bounds terms, plus
 * 48 per invalid term. Host buffers. */
int rcmvs_plane_cost_field(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                           int32_t ref_idx, const int32_t* srcs, int32_t n_src,
                           const float* planes, const float* hints, float* cost_out,
                           int32_t* hsum_out);

/* Number of plane_cost evaluations and 5-term window rows the last
 * rcmvs_scene_estimate_depth call performed (after gates and early aborts);
 * counted only when the RCMVS_COUNT environment variable is set at context
 * creation, else both are 0. */
int rcmvs_last_work(rcmvs_ctx* ctx, uint64_t* cost_evals, uint64_t* rows);

/* Per-kernel timing with CUDA events recorded on the context stream around
 * each launch of the stereo and fusion kernels.  enable != 0 starts a new
 * recording (dropping earlier spans); rcmvs_ctx_kernel_time synchronises and
 * returns the summed milliseconds and launch count of one kernel name
 * ("census_rays", "stereo_init", "stereo_pass", "stereo_gate",
 * "fuse_candidates", "fuse_reduce"). */
int rcmvs_ctx_timing(rcmvs_ctx* ctx, int enable);
int rcmvs_ctx_kernel_time(rcmvs_ctx* ctx, const char* name, double* ms_total, uint64_t* launches);

/* Converts n floats with the device's truncating float->int conversion, the
 * one the cost kernel uses for the reference's `as i32` (stereo.rs:205-206):
 * truncation toward zero, saturation, NaN -> 0.  Lets tests check those
 * semantics on the GPU.  Host buffers. */
int rcmvs_selftest_f2i(rcmvs_ctx* ctx, const float* in, int32_t n, int32_t* out);


/* ------------------------------------------- learned plane proposals */
/* No counterpart in the reference, which seeds every pixel with the plane
 * sweep.  A 6-layer 3x3 convolutional network (32 channels, ReLU; BF16
 * weights and activations, FP32 accumulation on the tensor cores) reads a
 * quarter-resolution input of 48 channels — a 32-plane census cost volume
 * (fronto-parallel planes at the centres of 32 equal inverse-depth bins,
 * mean Hamming fraction over a 3x3 window and the support views), the grey
 * image /255, 15 zeros — and predicts 16 channels per quarter pixel: t (the
 * inverse depth as a fraction of [1/zmax, 1/zmin]), a normal (3), a
 * confidence logit, 11 zeros.  Tensors are NHWC, BF16 unless noted. */
typedef struct rcmvs_net rcmvs_net;

/* Number of f32 parameters: for each layer W[9][cout][cin] then b[cout],
 * with (cin, cout) = (48,32), (32,32) x4, (32,16); padded entries are 0. */
uint64_t rcmvs_net_param_count(void);
/* params (nullable): initial parameters; NULL = He initialisation from seed. */
int rcmvs_net_create(rcmvs_ctx* ctx, const float* params, uint64_t seed, rcmvs_net** out);
void rcmvs_net_destroy(rcmvs_net* net);
int rcmvs_net_get_params(rcmvs_net* net, float* out);
/* Forward pass on device buffers: x_dev n*h*w*48 BF16 -> out_dev n*h*w*16 f32. */
int rcmvs_net_forward(rcmvs_ctx* ctx, rcmvs_net* net, const void* x_dev, int32_t n, int32_t h,
                      int32_t w, float* out_dev);
/* One training step on device buffers.  labels_dev: n*h*w*8 f32 = (t*, n*x,
 * n*y, n*z, valid, tolerance on t, 0, 0).  Loss per valid pixel:
 * |t - t*| + (1 - cos(n, n*)) + 0.1 BCE(sigmoid(logit), |t - t*| < tol).
 * apply != 0 takes an Adam step (lr); loss_out / grads_host (nullable)
 * receive the mean loss and its gradient (f32, parameter layout). */
int rcmvs_net_train_step(rcmvs_ctx* ctx, rcmvs_net* net, const void* x_dev,
                         const float* labels_dev, int32_t n, int32_t h, int32_t w, float lr,
                         int32_t apply, float* loss_out, float* grads_host);
/* Network input of each job's reference view (quarter resolution
 * (w/4)x(h/4), jobs back to back) into out_dev (BF16, 16-byte aligned). */
int rcmvs_scene_costvol(rcmvs_ctx* ctx, rcmvs_scene* scene, const rcmvs_job* jobs, int32_t n_jobs,
                        void* out_dev);
/* Stereo seeded by the network: a pixel whose prediction has confidence >=
 * conf_thr starts from the best of n_local planes with the predicted normal
 * and inverse depths spread over +-span/2 (fraction of the inverse-depth
 * range) around the prediction (plane_cost with the sweep's early-abort
 * hint; planes failing the stereo gates are skipped); the other pixels run
 * the plane sweep; then 2*max(sweeps,1) passes and the gate, as
 * rcmvs_scene_estimate_depth.  learned_pixels (nullable): pixels seeded by
 * the network. */
int rcmvs_scene_estimate_depth_learned(rcmvs_ctx* ctx, rcmvs_scene* scene, const rcmvs_job* jobs,
                                       int32_t n_jobs, const rcmvs_options* opts, rcmvs_net* net,
                                       float conf_thr, int32_t n_local, float span,
                                       uint64_t* learned_pixels);

/* rcmvs_scene_estimate_depth_learned with caller-given proposals in place of
 * the network's: pred holds, for each job in order, its reference view's
 * (w/4)*(h/4) quarter cells of 16 f32 (t, normal xyz, confidence logit, 11
 * unused; the layout rcmvs_net_forward writes), jobs back to back;
 * pred_on_device != 0 when pred is device memory.  A cell's confidence is
 * sigmoid(logit), tested as logit >= ln(conf_thr / (1 - conf_thr)). */
int rcmvs_scene_estimate_depth_seeded(rcmvs_ctx* ctx, rcmvs_scene* scene, const rcmvs_job* jobs,
                                      int32_t n_jobs, const rcmvs_options* opts, const float* pred,
                                      int32_t pred_on_device, float conf_thr, int32_t n_local,
                                      float span, uint64_t* learned_pixels);

/* rcmvs_run_mvs with stereo seeded by the network (arguments as
 * rcmvs_scene_estimate_depth_learned; opts->sweeps sweeps after the init). */
int rcmvs_run_mvs_learned(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views,
                          const rcmvs_sparse* sparse, const rcmvs_options* opts, rcmvs_net* net,
                          float conf_thr, int32_t n_local, float span,
                          const rcmvs_depth_out* depth_outs, rcmvs_points* out, rcmvs_stats* stats);

/* ------------------------------------------- allocation-free variant */
/* No counterpart in the reference: an `estimate_depth` for callers that may
 * not allocate device memory (an application whose GPU memory belongs to
 * another allocator, or a real-time loop that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree).  It makes no cudaMalloc/cudaFree
 * call and uses no allocating library routine: intermediates live in one
 * fixed __device__ array of RCMVS_NOALLOC_SCRATCH_BYTES (36.6 MiB), which a
 * device reserves when this entry point first runs there and holds until the
 * process exits (every device that loads the library, if modules load
 * eagerly).
 *   - views[i].gray are DEVICE pointers (w*h u8); rgb is ignored.
 *   - depth_dev / cost_dev are DEVICE buffers of w*h floats of the reference.
 *   - stream is a cudaStream_t (NULL = the legacy default stream); the call
 *     is asynchronous on it.  Results equal rcmvs_estimate_depth's bit for
 *     bit.
 *   - Each view at most RCMVS_NOALLOC_MAX_PIXELS pixels and at most
 *     RCMVS_NOALLOC_MAX_SOURCES sources, else RCMVS_E_LIMIT; bad arguments
 *     give RCMVS_E_ARG, a failed CUDA call RCMVS_E_CUDA (no message: there
 *     is no context).
 *   - Every call looks up the array's device address on the current device
 *     (cudaGetSymbolAddress, which allocates nothing); the first lookup on
 *     a device loads the library's module there, so make the first call on
 *     a device before any stream capture.
 *   - opts->flags may hold RCMVS_FLAG_ONE_CANDIDATE, RCMVS_FLAG_INIT_ONLY,
 *     RCMVS_FLAG_NO_SKIP_DUPLICATES and RCMVS_FLAG_NO_REPEAT_SKIP (this
 *     entry point never skips) and RCMVS_FLAG_SEED_AND_SWEEP (no effect
 *     here); the scheduling flags
 *     (PERSISTENT, CUDA_GRAPH, AUTOTUNE) give RCMVS_E_ARG.  The tile is
 *     tile_w x tile_h, default 8x8, as for rcmvs_estimate_depth.
 *   - All calls on a device share the array and leave its contents behind;
 *     calls whose GPU work overlaps (different streams or threads) race on
 *     it and must be serialised by the caller. */
#define RCMVS_NOALLOC_MAX_PIXELS 307200 /* 640 x 480 */
#define RCMVS_NOALLOC_MAX_SOURCES 4
#define RCMVS_NOALLOC_SCRATCH_BYTES 38416384
int rcmvs_estimate_depth_noalloc(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                                 const int32_t* srcs, int32_t n_src, double zmin, double zmax,
                                 const rcmvs_options* opts, float* depth_dev, float* cost_dev,
                                 void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RCMVS_H */
