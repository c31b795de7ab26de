// rcmvs_internal.cuh — device-side layouts and launcher declarations shared by
// the translation units of librcmvs (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/rcmvs.h"

namespace rcmvs {

// ---------------------------------------------------------------- layouts
// One view of a device-resident scene.  Per-pixel arrays of all views are
// concatenated; a view's pixels start at `off`.
struct DevView {
    int32_t w, h;
    int64_t off;
};

// One support view of a job, in the form the cost kernel reads (the
// SourceCtx of mvs/src/stereo.rs:84-96): relative pose and intrinsics in f32
// (cast from f64 on the host) and the census location.  20 words.
struct DevSrc {
    float rs[9];
    float ts[3];
    float f, cx, cy, k;
    int32_t w, h;
    int64_t off;  // pixel offset of the source view's census
};
static_assert(sizeof(DevSrc) == 80, "DevSrc layout");

// One estimate_depth job.  Tiles of all jobs of a launch are numbered
// consecutively; job j owns tiles [tile_base, tile_base + tiles).
struct DevJob {
    int32_t view, nsrc, w, h;
    int64_t off;        // pixel offset of the reference view
    float zmin, zmax;   // ws.zmin / ws.zmax (f32)
    float inv_min, inv_max;
    int32_t tiles_x, tiles_y;
    int32_t tile_base, tiles;
    int32_t tw, th;     // this job's tile shape (jobs of one launch may differ)
    DevSrc src[RCMVS_MAX_SOURCES];
};
static_assert(sizeof(DevJob) % 8 == 0, "DevJob layout");

// Plane of mvs/src/stereo.rs:24-31, split for 16-byte loads:
// float4 (nx, ny, nz, z) + float cost.  `d` (nullable) keeps, per pixel, the
// plane offset d the stored cost was computed with (z = d / (n . ray)); with
// it the pass kernel skips a propagation candidate that repeats the pixel's
// own plane bit for bit (see pass_kernel).  `flag` (nullable) holds one byte
// per pixel written by a pass: bit 0 = the pass wrote a new plane, bit 1 =
// a candidate beat the stored cost but its plane was refused (n . ray <=
// 0.05), so the stored cost is not the pass's best.  A pass that reads them
// (prev.flag set, `d` set) skips the propagation candidates that provably
// lose again (see pass_kernel); prev.flag is null for the first pass after
// an init.
struct PlaneBuf {
    float4* nz;   // (nx, ny, nz, z)
    float* cost;
    float* d = nullptr;
    uint8_t* flag = nullptr;
};

// Tile shape of one job's stereo launch (pixels per block = tw * th).
struct TileShape {
    int tw, th;
};

// Launch geometry of a stereo launch over the tiles of a job list.  Every
// job's tile has at most `nthr` pixels; blocks have `nthr` threads and
// `smem` bytes of dynamic shared memory (the largest tile's).  With `queue`
// set (a zeroed counter), the launch is persistent: a grid of resident blocks
// pulls tile indices from the counter until all `tiles` are taken;
// otherwise block b computes tile b.
struct LaunchGeom {
    int nthr;  // threads of a one-thread-per-pixel block (= the largest tile's pixels)
    size_t smem;
    int tiles;
    unsigned int* queue;
    int tpp = 1;  // threads per pixel of the passes: 1, or 5 (pass_split_kernel)
    bool stream = false;  // passes: pass_stream_kernel over the stream tiling (stream_geom)
    float4* scratch = nullptr;  // streamed passes: per-block scratch (stream_scratch_bytes)
    int scratch_blocks = 0;     // blocks the scratch holds (the launch uses at most this many)
};
// Streamed passes (pass_stream_kernel): tiles of a w x h view in the
// kernel's own tiling, and the geometry of a launch over `tiles` of them.
// The launch is always persistent (g.queue set) over at most
// stream_grid(g) blocks, each with its own slice of a device scratch of
// stream_scratch_bytes(blocks) bytes (its pixels' random candidates).
int stream_tiles(int w, int h);
LaunchGeom stream_geom(int tiles);
int stream_grid(const LaunchGeom& g);
size_t stream_scratch_bytes(int blocks);
// Threads of a split-pass block (5 lanes per pixel, 6 pixels per warp) for
// tiles of up to px pixels.
int split_threads(int px);

// ---------------------------------------------------------------- launchers
// Defined in census.cu and stereo.cu.  All are asynchronous on the given
// stream.  The stereo launchers run one kernel over every tile of a job list
// (job j owns tiles [job_start[j], job_start[j+1])).

// census + rays of every view (mvs/src/lib.rs:119-142, sfm-lite geom.rs:28-42)
// Stereo tile shapes: at most 256 pixels, a multiple of 32, shared memory
// within 48 KB; the default is opts' tile_w x tile_h, else 8x8.
bool tile_shape_ok(TileShape ts);
TileShape default_tile_shape(const rcmvs_options* opts);
// Tiles (blocks) the census kernel uses for a w x h view; a scene's views
// take consecutive tile ranges.
int census_tiles(int w, int h);
cudaError_t launch_census_rays(const DevView* d_views, const int32_t* d_tile_start, int n_views, int total_tiles,
                               const uint8_t* gray, uint64_t* census, float2* rays, const double* d_cams,
                               cudaStream_t st);
size_t stereo_smem_bytes(TileShape ts);
// Blocks a persistent launch of the pass kernel uses for geometry g.
int stereo_resident_grid(const LaunchGeom& g);
// Plane-sweep init (stereo.rs:247-269).  variant 0: row-step schedule;
// 1: one candidate at a time.  Bit-identical outputs.
cudaError_t launch_init(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g, int nh,
                        const uint64_t* census, const float2* rays, PlaneBuf out, unsigned long long* d_work,
                        cudaStream_t st, int variant);
// One Jacobi pass prev -> next (stereo.rs:271-371).
cudaError_t launch_pass(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g,
                        uint64_t pass, float sig_inv, float sig_n, const uint64_t* census, const float2* rays,
                        PlaneBuf prev, PlaneBuf next, unsigned long long* d_work, cudaStream_t st);
// Init seeded by the proposal network's predictions (no reference counterpart).
cudaError_t launch_init_learned(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g,
                                int nh, const uint64_t* census, const float2* rays, PlaneBuf out, const float* pred,
                                const int64_t* pred_off, float logit_thr, int n_local, float span, bool sweep_seeded,
                                unsigned long long* d_learned, cudaStream_t st);
// Texture/cost/range gate (stereo.rs:373-393); never persistent.
cudaError_t launch_gate(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g,
                        float cost_thr, const uint64_t* census, PlaneBuf planes, float* depth, float* cost,
                        float* normal, cudaStream_t st);
// Cost of a given plane field for one job (diagnostics / parity tests).
cudaError_t launch_cost_field(const DevJob* d_job, const int32_t* d_job_start, const LaunchGeom& g,
                              const uint64_t* census, const float2* rays, const float4* planes, const float* hints,
                              float* cost_out, int32_t* hsum_out, cudaStream_t st);
cudaError_t launch_f2i(const float* in, int n, int32_t* out, cudaStream_t st);

// Fusion (fuse.cu).  View arrays hold per-view f64 cameras/poses.
struct FuseView {
    int32_t w, h;
    int64_t off;
    int32_t has_depth;
    int32_t order_begin, order_end;
    int32_t is_ref;  // its pixels are checked (else it only serves as a source)
    double f, cx, cy, k;
    double R[9];
    double t[3];
};

struct FuseResult {
    uint64_t n_candidates;
    uint64_t n_points;
};

// Optional CUDA-event spans around kernel launches (per-kernel timing on
// the launching stream).  begin/end record an event pair named `name`.
struct SpanHook {
    void (*mark)(void* user, const char* name, int begin) = nullptr;
    void* user = nullptr;
    void begin(const char* n) const {
        if (mark) mark(user, n, 1);
    }
    void end(const char* n) const {
        if (mark) mark(user, n, 0);
    }
};

// Runs the whole device fusion; outputs stay in arena slots and are
// returned through d_xyz / d_rgb / d_ply.  See fuse.cu.
struct DeviceArena;
int fuse_device(DeviceArena& arena, const FuseView* h_views, int n_views, const int32_t* h_order,
                int n_order, const float* depth, const uint8_t* rgb, double cell, uint32_t min_consistent,
                double depth_diff, double reproj_px, double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply,
                FuseResult* res, cudaStream_t st, std::string* err, const SpanHook& hook);

// The two stages of fuse_device.  Candidates: the consistency check of the
// pixels of views with has_depth && is_ref; *d_cand gets the ascending
// global pixel indices of the candidates (n_cand of them) and *d_pts the
// per-pixel point buffer they index (3 doubles per global pixel).
int fuse_candidates_device(DeviceArena& arena, const FuseView* h_views, int n_views, const int32_t* h_order,
                           int n_order, const float* depth, uint32_t min_consistent, double depth_diff,
                           double reproj_px, const uint32_t** d_cand, uint32_t* n_cand, const double** d_pts,
                           cudaStream_t st, std::string* err, const SpanHook& hook);
// Voxel dedup of candidates cand[0..n_cand) in that order (indices into pts,
// 3 doubles each, and rgb, 3 bytes each).
int fuse_reduce_device(DeviceArena& arena, const uint32_t* d_cand, uint32_t n_cand, const double* pts,
                       const uint8_t* rgb, double cell, double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply,
                       uint64_t* n_points, cudaStream_t st, std::string* err, const SpanHook& hook);
// fuse_reduce_device over n host candidates (3 doubles + 3 bytes each),
// uploaded in the order given.
int fuse_reduce_host(DeviceArena& arena, const double* h_xyz, const uint8_t* h_rgb, uint64_t n, double cell,
                     double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply, uint64_t* n_points, cudaStream_t st,
                     std::string* err, const SpanHook& hook);
// The candidates' points and colours compacted in list order (device).
// fuse_reduce_device over n device-resident candidates (3 doubles + 3
// bytes each, caller memory), in the order given.
int fuse_reduce_devptr(DeviceArena& arena, const double* d_in_xyz, const uint8_t* d_in_rgb, uint64_t n, double cell,
                       double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply, uint64_t* n_points, cudaStream_t st,
                       std::string* err, const SpanHook& hook);
int fuse_gather_device(DeviceArena& arena, const uint32_t* d_cand, uint32_t n, const double* pts,
                       const uint8_t* rgb, double** d_xyz, uint8_t** d_rgb, cudaStream_t st, std::string* err);

// Grow-only device scratch memory owned by a context, carved into named
// slots so repeated calls reuse allocations.
struct DeviceArena {
    struct Slot {
        void* p = nullptr;
        size_t bytes = 0;
    };
    std::vector<Slot> slots;
    cudaError_t get(int slot, size_t bytes, void** out);
    void release();
};

}  // namespace rcmvs
