// ctx_internal.cuh — definitions of the opaque rcmvs_ctx / rcmvs_scene
// handles, shared by the translation units that implement the C ABI.
#pragma once

#include <string>
#include <vector>

#include "rcmvs_internal.cuh"

using rcmvs::DevView;
using rcmvs::DeviceArena;
using rcmvs::SpanHook;
using rcmvs::TileShape;

// per-pixel device buffers of a scene (rcmvs_scene, SpareScene::big)
constexpr int kSceneBig = 15;

struct rcmvs_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // rcmvs_run_mvs*: the views' RGB uploads run here, beside the stereo on
    // `stream` (RGB is read by fusion only); created on first use
    cudaStream_t upload = nullptr;
    std::string err;
    DeviceArena arena;
    bool count_work = false;
    unsigned long long* d_work = nullptr;
    uint64_t last_evals = 0, last_rows = 0;
    // autotuned tile shapes per resolution class, one thread count and one
    // threads-per-pixel of the passes for all
    std::vector<rcmvs_tune_entry> tuned;
    int tune_nthr = 0;
    int tune_tpp = 1;
    // per-kernel CUDA-event spans (rcmvs_ctx_timing)
    struct Span {
        std::string name;
        cudaEvent_t a, b;
    };
    bool timing = false;
    std::vector<Span> spans;
    // Device buffers and scratch arena of the last destroyed scene, adopted
    // by the next scene they are large enough for (rcmvs_scene_create), so
    // repeated rcmvs_run_mvs* calls on a workload allocate nothing.  Freed
    // with the context.  Order of `big`: gray, rgb, census, rays, plane_a,
    // plane_b, pcost_a, pcost_b, pd_a, pd_b, depth, cost, normal, pf_a, pf_b;
    // `small`: d_views, d_tile_start, d_cams.
    struct SpareScene {
        bool valid = false;
        size_t cap_px = 0;
        int cap_views = 0;
        void* big[kSceneBig] = {};
        void* small[3] = {};
        DeviceArena arena;
        // the learned path's quarter-resolution buffers, in the order of
        // rcmvs_scene's gray_q .. d_qblk_start, for scenes of at most
        // q_cap_px quarter pixels and q_cap_views views
        void* quarter[7] = {};
        size_t q_cap_px = 0;
        int q_cap_views = 0;
    } spare;
    // scenes created on this context and not yet destroyed; a context that
    // is destroyed first detaches them (they then free their own buffers)
    std::vector<rcmvs_scene*> live;
    SpanHook hook() {
        SpanHook h;
        if (timing) {
            h.mark = &rcmvs_ctx::mark_cb;
            h.user = this;
        }
        return h;
    }
    static void mark_cb(void* user, const char* name, int begin) {
        rcmvs_ctx* c = (rcmvs_ctx*)user;
        if (begin) {
            Span s;
            s.name = name;
            if (cudaEventCreate(&s.a) != cudaSuccess) return;
            if (cudaEventCreate(&s.b) != cudaSuccess) {
                cudaEventDestroy(s.a);
                return;
            }
            cudaEventRecord(s.a, c->stream);
            c->spans.push_back(s);
        } else if (!c->spans.empty() && c->spans.back().name == name) {
            cudaEventRecord(c->spans.back().b, c->stream);
        }
    }
    void clear_spans() {
        for (auto& s : spans) {
            cudaEventDestroy(s.a);
            cudaEventDestroy(s.b);
        }
        spans.clear();
    }
};

struct HostCam {
    double f, cx, cy, k;
    double R[9], t[3];
};

struct rcmvs_scene {
    rcmvs_ctx* ctx = nullptr;
    int n_views = 0;
    int64_t n_px = 0;
    size_t cap_px = 0;  // pixels / views the device buffers hold (0 until allocated)
    int cap_views = 0;
    std::vector<DevView> views;
    std::vector<HostCam> cams;
    std::vector<char> has_depth;
    bool has_rgb = false;
    int census_tiles = 0;
    // device buffers
    uint8_t* gray = nullptr;
    uint8_t* rgb = nullptr;
    uint64_t* census = nullptr;
    float2* rays = nullptr;
    float4* plane_a = nullptr;
    float4* plane_b = nullptr;
    float* pcost_a = nullptr;
    float* pcost_b = nullptr;
    float* pd_a = nullptr;  // plane offsets d (PlaneBuf::d)
    float* pd_b = nullptr;
    uint8_t* pf_a = nullptr;  // per-pixel pass flags (PlaneBuf::flag)
    uint8_t* pf_b = nullptr;
    float* depth = nullptr;
    float* cost = nullptr;
    float* normal = nullptr;
    DevView* d_views = nullptr;
    int32_t* d_tile_start = nullptr;
    double* d_cams = nullptr;
    DeviceArena arena;  // jobs + fusion scratch/outputs
    uint64_t n_points = 0;
    uint64_t n_candidates = 0;
    double* d_pts_xyz = nullptr;
    uint8_t* d_pts_rgb = nullptr;
    uint8_t* d_ply = nullptr;
    // candidates kept by rcmvs_scene_fuse_candidates_device (arena memory)
    uint64_t n_kept = 0;
    const double* d_kept_xyz = nullptr;
    const uint8_t* d_kept_rgb = nullptr;
    // quarter-resolution copies for learned proposals (allocated on first use)
    bool have_quarter = false;
    std::vector<DevView> qviews;
    uint8_t* gray_q = nullptr;
    uint64_t* census_q = nullptr;
    float2* rays_q = nullptr;
    DevView* d_qviews = nullptr;
    int32_t* d_qtile_start = nullptr;
    double* d_qcams = nullptr;
    int32_t* d_qblk_start = nullptr;
    int qcensus_tiles = 0, qblocks = 0;
    int64_t nq_px = 0;
    size_t q_cap_px = 0;  // capacity of the quarter buffers (pixels, views)
    int q_cap_views = 0;
    // the last captured stereo schedule (RCMVS_FLAG_CUDA_GRAPH) and its key
    cudaGraphExec_t graph = nullptr;
    std::vector<unsigned char> graph_key;
};

namespace rcmvs {

// Arena slots of a scene shared by the translation units (the others are
// private to capi.cu 2-10, fuse.cu 16-37 and 70-74, learned_api.cu 40-47, depthvis.cu 50-55,
// resize.cu 60-68, sift.cu 80-159 and match.cu 160-167).
constexpr int kSlotJobs = 0, kSlotJobStart = 1, kSlotQueue = 11, kSlotTuneJobs = 12, kSlotTuneStart = 13,
              kSlotStreamStart = 14, kSlotStreamScratch = 15;

// resize.cu: argument and size checks of a resize, and the resize itself
// on device buffers (d_gray mw*mh, d_rgb mw*mh*3), queued on the context's
// stream; *d_err (null when no resize ran) is a device flag, non-zero if a
// tap table overflowed.  Uses context arena slots 61 and 64-68.
int resize_check(rcmvs_ctx* ctx, int w, int h, int channels, int mw, int mh);
int resize_device(rcmvs_ctx* ctx, const uint8_t* d_in, int w, int h, int channels, int mw, int mh, uint8_t* d_gray,
                  uint8_t* d_rgb, const int** d_err);

// mvs/src/stereo.rs:131-132: source pose relative to the reference, f64
// products cast to f32.
void rel_pose(const HostCam& r, const HostCam& s, float* rs, float* ts);
// mvs/src/stereo.rs:114-151: one job's device descriptor (relative poses in
// f64 cast to f32, source intrinsics and census offsets), tile shape ts.
void fill_job(const rcmvs_scene* sc, int ref, const int32_t* srcs, int n_src, double zmin, double zmax, TileShape ts,
              DevJob& J);

// One stereo batch as launched: jobs in launch order (longest tiles first),
// their tile starts, the caller's index of each, and the launch geometry.
struct StereoBatch {
    std::vector<DevJob> jobs;
    std::vector<int32_t> start;  // n_jobs + 1
    std::vector<int> order;      // launch position -> caller's job index
    LaunchGeom geom{};
    // streamed passes (pass_stream_kernel, the default): the jobs' tile starts
    // in that kernel's tiling (n_jobs + 1) and its launch geometry
    bool stream = false;
    std::vector<int32_t> sstart;
    LaunchGeom sgeom{};
};

// The launch schedule of a batch: init -> n_passes Jacobi passes -> gate.
struct Schedule {
    enum Init { ROWS = 0, ONE_CANDIDATE = 1, LEARNED = 2, TABLE = 3 } init = ROWS;
    int nh = 64;
    uint64_t n_passes = 12;
    float cost_thr = 0.38f;
    bool persistent = false;
    bool graph = false;
    bool skip_duplicates = true;  // PlaneBuf::d on: skip repeated propagation candidates
    bool repeat_skip = true;      // PlaneBuf::flag on (with skip_duplicates): skip candidates that lost before
    unsigned long long* d_work = nullptr;  // work counters (zeroed by the caller)
    // learned init
    const float* pred = nullptr;
    const int64_t* pred_off = nullptr;  // per launch position
    float logit_thr = 0.f;  // confident iff logit >= logit_thr
    int n_local = 1;
    float span = 0.f;
    bool sweep_seeded = false;  // seeded pixels also run the plane sweep (RCMVS_FLAG_SEED_AND_SWEEP)
    unsigned long long* d_learned = nullptr;  // zeroed inside the schedule
};

// Validates shapes, looks up (and with RCMVS_FLAG_AUTOTUNE, first tunes)
// per-class shapes, orders jobs and fills b.  Returns an RCMVS_* code.
int build_batch(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, const rcmvs_options* opts,
                StereoBatch& b);
// Uploads b's job table and runs the schedule on the context stream
// (asynchronous).  Returns an RCMVS_* code.
int run_batch(rcmvs_ctx* ctx, rcmvs_scene* sc, const StereoBatch& b, const Schedule& s);
// Drops the scene's cached graph.
void drop_graph(rcmvs_scene* sc);

}  // namespace rcmvs

