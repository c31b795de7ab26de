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
    DevSrc src[RCMVS_MAX_SOURCES];
};

// Plane of mvs/src/stereo.rs:24-31, split for 16-byte loads:
// float4 (nx, ny, nz, z) + float cost.
struct PlaneBuf {
    float4* nz;   // (nx, ny, nz, z)
    float* cost;
};

// Kernel launch geometry of the stereo kernels.
struct TileShape {
    int tw, th;
};

// ---------------------------------------------------------------- launchers
// Declared (and documented) where they are used, in capi.cu; defined in
// census.cu and stereo.cu.  All are asynchronous on the given stream.

// Fusion (fuse.cu).  View arrays hold per-view f64 cameras/poses.
struct FuseView {
    int32_t w, h;
    int64_t off;
    int32_t has_depth;
    int32_t order_begin, order_end;
    int32_t pad;
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
