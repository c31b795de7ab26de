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

struct rcmvs_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    DeviceArena arena;
    bool count_work = false;
    unsigned long long* d_work = nullptr;
    uint64_t last_evals = 0, last_rows = 0;
    TileShape configured{0, 0};
    // per-kernel CUDA-event spans (rcmvs_ctx_timing)
    struct Span {
        std::string name;
        cudaEvent_t a, b;
    };
    bool timing = false;
    std::vector<Span> spans;
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
};

