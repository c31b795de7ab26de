// capi.cu — the C ABI of librcmvs (include/rcmvs.h): contexts, device-resident
// scenes, the host-buffer entry points that stand in for the reference `mvs`
// crate, the run_mvs host glue and the PLY writer.
#include <algorithm>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "rcmvs_internal.cuh"

namespace rcmvs {

cudaError_t DeviceArena::get(int slot, size_t bytes, void** out) {
    if ((int)slots.size() <= slot) slots.resize(slot + 1);
    Slot& s = slots[slot];
    if (bytes == 0) bytes = 16;
    if (s.bytes < bytes) {
        if (s.p) {
            cudaError_t e = cudaFree(s.p);
            if (e != cudaSuccess) return e;
            s.p = nullptr;
            s.bytes = 0;
        }
        size_t nb = std::max(bytes, s.bytes + s.bytes / 4);
        cudaError_t e = cudaMalloc(&s.p, nb);
        if (e != cudaSuccess) {
            s.p = nullptr;
            return e;
        }
        s.bytes = nb;
    }
    *out = s.p;
    return cudaSuccess;
}

void DeviceArena::release() {
    for (auto& s : slots)
        if (s.p) cudaFree(s.p);
    slots.clear();
}

}  // namespace rcmvs

using namespace rcmvs;

#include "ctx_internal.cuh"
#include "learned.cuh"

namespace {

void free_spare(rcmvs_ctx* ctx);

enum { S_JOBS = kSlotJobs, S_JOBSTART = kSlotJobStart, S_CGRAY = 2, S_CCEN = 3, S_FIELD_PL = 4, S_FIELD_H = 5,
       S_FIELD_C = 6, S_FIELD_HS = 7, S_F2I = 8 };

int fail(rcmvs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,    \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

bool finite(double x) { return std::isfinite(x); }

int check_view(rcmvs_ctx* ctx, const rcmvs_view& v, int i, const rcmvs_options* opts) {
    if (v.w <= 0 || v.h <= 0 || !v.gray)
        return fail(ctx, RCMVS_E_ARG, "view " + std::to_string(i) + ": bad size or null gray");
    if (v.w > (1 << 23) || v.h > (1 << 23))  // the stereo kernels' exact index arithmetic
        return fail(ctx, RCMVS_E_LIMIT, "view " + std::to_string(i) + ": a side longer than 2^23 pixels");
    if (!(finite(v.f) && v.f != 0.0 && finite(v.cx) && finite(v.cy) && finite(v.k)))
        return fail(ctx, RCMVS_E_ARG, "view " + std::to_string(i) + ": non-finite or zero intrinsics");
    for (int q = 0; q < 9; ++q)
        if (!finite(v.R[q])) return fail(ctx, RCMVS_E_ARG, "view " + std::to_string(i) + ": non-finite pose");
    for (int q = 0; q < 3; ++q)
        if (!finite(v.t[q])) return fail(ctx, RCMVS_E_ARG, "view " + std::to_string(i) + ": non-finite pose");
    if (opts && (uint32_t)std::max(v.w, v.h) > opts->max_dim)
        return fail(ctx, RCMVS_E_ARG,
                    "view " + std::to_string(i) + ": long side exceeds max_dim (views must be given at the "
                    "stereo working resolution)");
    return RCMVS_OK;
}

int validate_jobs(rcmvs_ctx* ctx, int n_views, const rcmvs_job* jobs, int n_jobs) {
    if (n_jobs < 0 || (n_jobs > 0 && !jobs)) return fail(ctx, RCMVS_E_ARG, "bad job list");
    std::vector<char> seen(n_views, 0);
    for (int j = 0; j < n_jobs; ++j) {
        const rcmvs_job& b = jobs[j];
        if (b.ref_idx < 0 || b.ref_idx >= n_views) return fail(ctx, RCMVS_E_ARG, "job ref_idx out of range");
        if (seen[b.ref_idx]) return fail(ctx, RCMVS_E_ARG, "two jobs share a reference view");
        seen[b.ref_idx] = 1;
        if (b.n_src < 0 || (b.n_src > 0 && !b.srcs)) return fail(ctx, RCMVS_E_ARG, "bad source list");
        if (b.n_src > RCMVS_MAX_SOURCES)
            return fail(ctx, RCMVS_E_LIMIT, "more than RCMVS_MAX_SOURCES support views in one job");
        for (int s = 0; s < b.n_src; ++s)
            if (b.srcs[s] < 0 || b.srcs[s] >= n_views) return fail(ctx, RCMVS_E_ARG, "source index out of range");
        if (!(finite(b.zmin) && finite(b.zmax) && b.zmin > 0.0 && b.zmax > 0.0))
            return fail(ctx, RCMVS_E_ARG, "depth range must be finite and positive");
    }
    return RCMVS_OK;
}

}  // namespace

// ================================================================ context
extern "C" {

const char* rcmvs_version(void) { return "rcmvs 0.1 (sm_100a)"; }

uint64_t rcmvs_pass_count(const rcmvs_options* o) {
    if (!o || (o->flags & RCMVS_FLAG_INIT_ONLY)) return 0;
    if (o->passes) return o->passes;
    return (uint64_t)(o->sweeps > 1u ? o->sweeps : 1u) * 2u;
}

void rcmvs_options_default(rcmvs_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_dim = 900;  // mvs/src/lib.rs:56-70
    o->num_sources = 3;
    o->sweeps = 4;
    o->num_hyp = 48;
    o->min_consistent = 2;
    o->depth_diff = 0.03;
    o->cost_thr = 0.38f;
    o->voxel_rel = 0.0015;
    o->save_depth_vis = 0;
}

int rcmvs_ctx_create(int device, rcmvs_ctx** out) {
    if (!out) return RCMVS_E_ARG;
    *out = nullptr;
    rcmvs_ctx* ctx = new rcmvs_ctx();
    ctx->device = device;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device < 0 || device >= n) {
        delete ctx;
        return RCMVS_E_CUDA;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
        delete ctx;
        return RCMVS_E_CUDA;  // built for sm_100a only
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) {
        delete ctx;
        return RCMVS_E_CUDA;
    }
    const char* cw = std::getenv("RCMVS_COUNT");
    ctx->count_work = cw && cw[0] && cw[0] != '0';
    if (ctx->count_work) {
        if (cudaMalloc(&ctx->d_work, 2 * sizeof(unsigned long long)) != cudaSuccess) {
            cudaStreamDestroy(ctx->stream);
            delete ctx;
            return RCMVS_E_NOMEM;
        }
    }
    *out = ctx;
    return RCMVS_OK;
}

void rcmvs_ctx_destroy(rcmvs_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->arena.release();
    free_spare(ctx);
    for (rcmvs_scene* sc : ctx->live) sc->ctx = nullptr;
    ctx->clear_spans();
    if (ctx->d_work) cudaFree(ctx->d_work);
    if (ctx->upload) {
        cudaStreamSynchronize(ctx->upload);
        cudaStreamDestroy(ctx->upload);
    }
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* rcmvs_last_error(const rcmvs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* rcmvs_ctx_stream(rcmvs_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int rcmvs_diag_wait_timeout(rcmvs_ctx* ctx, uint64_t limit_ns) {
    if (!ctx) return RCMVS_E_ARG;
    if (limit_ns < 1000 || limit_ns > 1000000000ull) return fail(ctx, RCMVS_E_ARG, "limit_ns must be 1 us .. 1 s");
    CK(cudaSetDevice(ctx->device));
    CK(rcmvs::launch_wait_probe(limit_ns, ctx->stream));
    return RCMVS_OK;
}

int rcmvs_ctx_synchronize(rcmvs_ctx* ctx) {
    if (!ctx) return RCMVS_E_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    const int f = rcmvs::tc_fault_take();
    if (f) return fail(ctx, RCMVS_E_CUDA, f > 0 ? "a tensor-core kernel timed out waiting for its MMAs"
                                                 : "could not read the tensor-core fault word");
    return RCMVS_OK;
}

void rcmvs_points_free(rcmvs_points* p) {
    if (!p) return;
    std::free(p->xyz);
    std::free(p->rgb);
    p->xyz = nullptr;
    p->rgb = nullptr;
    p->n = 0;
}

// ================================================================ scene
}  // extern "C"

namespace {

void** scene_big(rcmvs_scene* sc, int i) {
    void** m[kSceneBig] = {(void**)&sc->gray,    (void**)&sc->rgb,     (void**)&sc->census, (void**)&sc->rays,
                           (void**)&sc->plane_a, (void**)&sc->plane_b, (void**)&sc->pcost_a, (void**)&sc->pcost_b,
                           (void**)&sc->pd_a,    (void**)&sc->pd_b,    (void**)&sc->depth,   (void**)&sc->cost,
                           (void**)&sc->normal,  (void**)&sc->pf_a,    (void**)&sc->pf_b};
    return m[i];
}

void** scene_small(rcmvs_scene* sc, int i) {
    void** m[3] = {(void**)&sc->d_views, (void**)&sc->d_tile_start, (void**)&sc->d_cams};
    return m[i];
}

void free_spare(rcmvs_ctx* ctx) {
    rcmvs_ctx::SpareScene& s = ctx->spare;
    for (void*& p : s.big) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    for (void*& p : s.small) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    s.arena.release();
    s.valid = false;
    s.cap_px = 0;
    s.cap_views = 0;
    for (void*& p : s.quarter) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    s.q_cap_px = 0;
    s.q_cap_views = 0;
}

}  // namespace

extern "C" {

void rcmvs_scene_destroy(rcmvs_scene* sc) {
    if (!sc) return;
    if (sc->ctx) {
        cudaSetDevice(sc->ctx->device);
        cudaStreamSynchronize(sc->ctx->stream);
        auto& live = sc->ctx->live;
        live.erase(std::remove(live.begin(), live.end(), sc), live.end());
    }
    void* quarter[7] = {sc->gray_q, sc->census_q, sc->rays_q, sc->d_qviews, sc->d_qtile_start, sc->d_qcams,
                        sc->d_qblk_start};
    drop_graph(sc);
    if (sc->ctx && sc->cap_px > 0) {
        // keep the buffers for the context's next scene
        free_spare(sc->ctx);
        rcmvs_ctx::SpareScene& s = sc->ctx->spare;
        for (int i = 0; i < kSceneBig; ++i) s.big[i] = *scene_big(sc, i);
        for (int i = 0; i < 3; ++i) s.small[i] = *scene_small(sc, i);
        s.arena.slots = std::move(sc->arena.slots);
        sc->arena.slots.clear();
        s.cap_px = sc->cap_px;
        s.cap_views = sc->cap_views;
        s.valid = true;
        for (int i = 0; i < 7; ++i) s.quarter[i] = quarter[i];
        s.q_cap_px = sc->q_cap_px;
        s.q_cap_views = sc->q_cap_views;
    } else {
        for (void* p : quarter)
            if (p) cudaFree(p);
        for (int i = 0; i < kSceneBig; ++i)
            if (*scene_big(sc, i)) cudaFree(*scene_big(sc, i));
        for (int i = 0; i < 3; ++i)
            if (*scene_small(sc, i)) cudaFree(*scene_small(sc, i));
        sc->arena.release();
    }
    delete sc;
}

int rcmvs_scene_prepare(rcmvs_ctx* ctx, rcmvs_scene* sc);

// rcmvs_scene_create; with `rgb_stream` set, the RGB uploads go on that
// stream instead (after the work already on ctx->stream) and `rgb_done` is
// recorded after them: the caller makes fusion wait for it and waits for it
// before the scene is destroyed or the host views may be released.
static int scene_create(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, rcmvs_scene** out,
                        cudaStream_t rgb_stream, cudaEvent_t rgb_done);

int rcmvs_scene_create(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, rcmvs_scene** out) {
    return scene_create(ctx, views, n_views, out, nullptr, nullptr);
}

static int scene_create(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, rcmvs_scene** out,
                        cudaStream_t rgb_stream, cudaEvent_t rgb_done) {
    if (!ctx || !views || n_views <= 0 || !out) return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_create: bad argument");
    *out = nullptr;
    for (int i = 0; i < n_views; ++i) {
        int rc = check_view(ctx, views[i], i, nullptr);
        if (rc) return rc;
    }
    CK(cudaSetDevice(ctx->device));
    rcmvs_scene* sc = new rcmvs_scene();
    sc->ctx = ctx;
    ctx->live.push_back(sc);
    sc->n_views = n_views;
    sc->has_rgb = true;
    int64_t off = 0;
    std::vector<int32_t> tile_start;
    int tiles = 0;
    for (int i = 0; i < n_views; ++i) {
        const rcmvs_view& v = views[i];
        sc->views.push_back(DevView{v.w, v.h, off});
        HostCam c;
        c.f = v.f;
        c.cx = v.cx;
        c.cy = v.cy;
        c.k = v.k;
        std::memcpy(c.R, v.R, sizeof(c.R));
        std::memcpy(c.t, v.t, sizeof(c.t));
        sc->cams.push_back(c);
        if (!v.rgb) sc->has_rgb = false;
        tile_start.push_back(tiles);
        tiles += census_tiles(v.w, v.h);
        off += (int64_t)v.w * v.h;
    }
    tile_start.push_back(tiles);
    sc->census_tiles = tiles;
    sc->n_px = off;
    sc->has_depth.assign(n_views, 0);
    const size_t np = (size_t)off;
    auto alloc = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes); };
    cudaError_t e = cudaSuccess;
    rcmvs_ctx::SpareScene& spare = ctx->spare;
    if (spare.valid && spare.cap_px >= np && spare.cap_views >= n_views && (spare.big[1] || !sc->has_rgb)) {
        // the previous scene's buffers and scratch: every one is written before it is read
        for (int i = 0; i < kSceneBig; ++i) *scene_big(sc, i) = spare.big[i];
        for (int i = 0; i < 3; ++i) *scene_small(sc, i) = spare.small[i];
        sc->arena.slots = std::move(spare.arena.slots);
        spare.arena.slots.clear();
        sc->cap_px = spare.cap_px;
        sc->cap_views = spare.cap_views;
        for (void*& p : spare.big) p = nullptr;
        for (void*& p : spare.small) p = nullptr;
        spare.valid = false;
    } else {
    if (!e) e = alloc((void**)&sc->gray, np);
    if (!e && sc->has_rgb) e = alloc((void**)&sc->rgb, 3 * np);
    if (!e) e = alloc((void**)&sc->census, 8 * np);
    if (!e) e = alloc((void**)&sc->rays, 8 * np);
    if (!e) e = alloc((void**)&sc->plane_a, 16 * np);
    if (!e) e = alloc((void**)&sc->plane_b, 16 * np);
    if (!e) e = alloc((void**)&sc->pcost_a, 4 * np);
    if (!e) e = alloc((void**)&sc->pcost_b, 4 * np);
    if (!e) e = alloc((void**)&sc->pd_a, 4 * np);
    if (!e) e = alloc((void**)&sc->pd_b, 4 * np);
    if (!e) e = alloc((void**)&sc->pf_a, np);
    if (!e) e = alloc((void**)&sc->pf_b, np);
    if (!e) e = alloc((void**)&sc->depth, 4 * np);
    if (!e) e = alloc((void**)&sc->cost, 4 * np);
    if (!e) e = alloc((void**)&sc->normal, 12 * np);
    if (!e) e = alloc((void**)&sc->d_views, sizeof(DevView) * n_views);
    if (!e) e = alloc((void**)&sc->d_tile_start, sizeof(int32_t) * (n_views + 1));
    if (!e) e = alloc((void**)&sc->d_cams, sizeof(double) * 4 * n_views);
    if (!e) {
        sc->cap_px = np;
        sc->cap_views = n_views;
    }
    }
    if (e) {
        rcmvs_scene_destroy(sc);
        return fail(ctx, e == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,
                    std::string("rcmvs_scene_create: ") + cudaGetErrorString(e));
    }
    std::vector<double> cams4;
    for (auto& c : sc->cams) cams4.insert(cams4.end(), {c.f, c.cx, c.cy, c.k});
    cudaStream_t st = ctx->stream;
    cudaStream_t rst = rgb_stream ? rgb_stream : st;
    if (rgb_stream) {  // adopted buffers may still be read by work queued on st
        if (!e) e = cudaEventRecord(rgb_done, st);
        if (!e) e = cudaStreamWaitEvent(rgb_stream, rgb_done, 0);
    }
    for (int i = 0; i < n_views && !e; ++i) {
        const size_t n = (size_t)views[i].w * views[i].h;
        e = cudaMemcpyAsync(sc->gray + sc->views[i].off, views[i].gray, n, cudaMemcpyHostToDevice, st);
    }
    for (int i = 0; i < n_views && !e && sc->has_rgb; ++i) {
        const size_t n = (size_t)views[i].w * views[i].h;
        e = cudaMemcpyAsync(sc->rgb + 3 * sc->views[i].off, views[i].rgb, 3 * n, cudaMemcpyHostToDevice, rst);
    }
    if (!e && rgb_stream) e = cudaEventRecord(rgb_done, rgb_stream);
    if (!e) e = cudaMemcpyAsync(sc->d_views, sc->views.data(), sizeof(DevView) * n_views, cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemcpyAsync(sc->d_tile_start, tile_start.data(), sizeof(int32_t) * (n_views + 1),
                                cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemcpyAsync(sc->d_cams, cams4.data(), sizeof(double) * cams4.size(), cudaMemcpyHostToDevice, st);
    // Callers of rcmvs_scene_create may release their views on return, so
    // the uploads finish first.  run_mvs keeps its views until it returns
    // and synchronises there, so its RGB uploads and the census overlap the
    // host plan glue.  (A copy from the pageable host vectors above waits
    // for the stream's earlier work, the grey uploads, and returns once its
    // source has been staged.)
    if (!e && !rgb_stream) e = cudaStreamSynchronize(st);
    if (e) {
        if (rgb_stream) cudaStreamSynchronize(rgb_stream);  // no upload into a released buffer
        rcmvs_scene_destroy(sc);
        return fail(ctx, RCMVS_E_CUDA, std::string("rcmvs_scene_create: ") + cudaGetErrorString(e));
    }
    int rc = rcmvs_scene_prepare(ctx, sc);
    if (rc) {
        if (rgb_stream) cudaStreamSynchronize(rgb_stream);
        rcmvs_scene_destroy(sc);
        return rc;
    }
    *out = sc;
    return RCMVS_OK;
}

// census + rays of every view (kernel a).  Asynchronous.
int rcmvs_scene_prepare(rcmvs_ctx* ctx, rcmvs_scene* sc) {
    if (!ctx || !sc) return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_prepare: bad argument");
    CK(cudaSetDevice(ctx->device));
    const SpanHook hk = ctx->hook();
    hk.begin("census_rays");
    CK(launch_census_rays(sc->d_views, sc->d_tile_start, sc->n_views, sc->census_tiles, sc->gray, sc->census,
                          sc->rays, sc->d_cams, ctx->stream));
    hk.end("census_rays");
    return RCMVS_OK;
}

int rcmvs_scene_estimate_depth(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int32_t n_jobs,
                               const rcmvs_options* opts) {
    if (!ctx || !sc || !opts) return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_estimate_depth: bad argument");
    if (sc->ctx != ctx) return fail(ctx, RCMVS_E_ARG, "scene belongs to another context");
    int rc = validate_jobs(ctx, sc->n_views, jobs, n_jobs);
    if (rc) return rc;
    for (int j = 0; j < n_jobs; ++j) {
        const DevView& V = sc->views[jobs[j].ref_idx];
        if ((uint32_t)std::max(V.w, V.h) > opts->max_dim)
            return fail(ctx, RCMVS_E_ARG, "reference view long side exceeds max_dim");
    }
    constexpr uint32_t kFlags = RCMVS_FLAG_ONE_CANDIDATE | RCMVS_FLAG_PERSISTENT | RCMVS_FLAG_CUDA_GRAPH |
                                RCMVS_FLAG_AUTOTUNE | RCMVS_FLAG_NO_SKIP_DUPLICATES | RCMVS_FLAG_INIT_ONLY |
                                RCMVS_FLAG_SEED_AND_SWEEP |  // only affects the learned init
                                RCMVS_FLAG_ROW_STEP_INIT | RCMVS_FLAG_NO_REPEAT_SKIP | RCMVS_FLAG_LOCKSTEP_PASSES;
    if (opts->flags & ~kFlags) return fail(ctx, RCMVS_E_ARG, "unknown bits in opts->flags");
    if (opts->passes > RCMVS_MAX_PASSES) return fail(ctx, RCMVS_E_ARG, "opts->passes above RCMVS_MAX_PASSES");
    if (n_jobs == 0) return RCMVS_OK;
    CK(cudaSetDevice(ctx->device));
    StereoBatch batch;
    rc = build_batch(ctx, sc, jobs, n_jobs, opts, batch);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    unsigned long long* dw = ctx->count_work ? ctx->d_work : nullptr;
    if (dw) CK(cudaMemsetAsync(dw, 0, 2 * sizeof(unsigned long long), st));
    Schedule s;
    s.init = (opts->flags & RCMVS_FLAG_ONE_CANDIDATE)  ? Schedule::ONE_CANDIDATE
             : (opts->flags & RCMVS_FLAG_ROW_STEP_INIT) ? Schedule::ROWS
                                                        : Schedule::TABLE;
    s.nh = (int)std::max<uint32_t>(opts->num_hyp, 2u);
    s.n_passes = rcmvs_pass_count(opts);
    s.cost_thr = opts->cost_thr;
    s.persistent = (opts->flags & RCMVS_FLAG_PERSISTENT) != 0;
    s.graph = (opts->flags & RCMVS_FLAG_CUDA_GRAPH) != 0;
    s.skip_duplicates = !(opts->flags & RCMVS_FLAG_NO_SKIP_DUPLICATES);
    s.repeat_skip = !(opts->flags & RCMVS_FLAG_NO_REPEAT_SKIP);
    s.d_work = dw;
    rc = run_batch(ctx, sc, batch, s);
    if (rc) return rc;
    for (int j = 0; j < n_jobs; ++j) sc->has_depth[jobs[j].ref_idx] = 1;
    if (dw) {
        unsigned long long h[2];
        CK(cudaMemcpyAsync(h, dw, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ctx->last_evals = h[0];
        ctx->last_rows = h[1];
    }
    return RCMVS_OK;
}

int rcmvs_ctx_timing(rcmvs_ctx* ctx, int enable) {
    if (!ctx) return RCMVS_E_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->clear_spans();
    ctx->timing = enable != 0;
    return RCMVS_OK;
}

int rcmvs_ctx_kernel_time(rcmvs_ctx* ctx, const char* name, double* ms_total, uint64_t* launches) {
    if (!ctx || !name || !ms_total || !launches) return RCMVS_E_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    double t = 0.0;
    uint64_t n = 0;
    for (auto& s : ctx->spans) {
        if (s.name != name) continue;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, s.a, s.b));
        t += ms;
        ++n;
    }
    *ms_total = t;
    *launches = n;
    return RCMVS_OK;
}

int rcmvs_last_work(rcmvs_ctx* ctx, uint64_t* evals, uint64_t* rows) {
    if (!ctx || !evals || !rows) return RCMVS_E_ARG;
    *evals = ctx->count_work ? ctx->last_evals : 0;
    *rows = ctx->count_work ? ctx->last_rows : 0;
    return RCMVS_OK;
}

int rcmvs_scene_get_depth(rcmvs_ctx* ctx, rcmvs_scene* sc, int32_t view, float* depth, float* cost, float* normal) {
    if (!ctx || !sc || view < 0 || view >= sc->n_views) return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_get_depth: bad argument");
    if (!sc->has_depth[view]) return fail(ctx, RCMVS_E_STATE, "view has no depth map");
    CK(cudaSetDevice(ctx->device));
    const DevView& V = sc->views[view];
    const size_t n = (size_t)V.w * V.h;
    cudaStream_t st = ctx->stream;
    if (depth) CK(cudaMemcpyAsync(depth, sc->depth + V.off, 4 * n, cudaMemcpyDeviceToHost, st));
    if (cost) CK(cudaMemcpyAsync(cost, sc->cost + V.off, 4 * n, cudaMemcpyDeviceToHost, st));
    if (normal) CK(cudaMemcpyAsync(normal, sc->normal + 3 * V.off, 12 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return RCMVS_OK;
}

int rcmvs_scene_depth_to_device(rcmvs_ctx* ctx, rcmvs_scene* sc, int32_t view, float* depth_dev) {
    if (!ctx || !sc || view < 0 || view >= sc->n_views || !depth_dev)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_depth_to_device: bad argument");
    if (!sc->has_depth[view]) return fail(ctx, RCMVS_E_STATE, "view has no depth map");
    CK(cudaSetDevice(ctx->device));
    const DevView& V = sc->views[view];
    CK(cudaMemcpyAsync(depth_dev, sc->depth + V.off, 4 * (size_t)V.w * V.h, cudaMemcpyDeviceToDevice, ctx->stream));
    return RCMVS_OK;
}

int rcmvs_scene_set_depth(rcmvs_ctx* ctx, rcmvs_scene* sc, int32_t view, const float* depth, int32_t on_device) {
    if (!ctx || !sc || view < 0 || view >= sc->n_views || !depth)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_set_depth: bad argument");
    CK(cudaSetDevice(ctx->device));
    const DevView& V = sc->views[view];
    CK(cudaMemcpyAsync(sc->depth + V.off, depth, 4 * (size_t)V.w * V.h,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    if (!on_device) CK(cudaStreamSynchronize(ctx->stream));  // the host buffer may go away on return
    sc->has_depth[view] = 1;
    return RCMVS_OK;
}

int rcmvs_scene_get_census(rcmvs_ctx* ctx, rcmvs_scene* sc, int32_t view, uint64_t* census) {
    if (!ctx || !sc || view < 0 || view >= sc->n_views || !census)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_get_census: bad argument");
    CK(cudaSetDevice(ctx->device));
    const DevView& V = sc->views[view];
    CK(cudaMemcpyAsync(census, sc->census + V.off, 8 * (size_t)V.w * V.h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return RCMVS_OK;
}

}  // extern "C"

namespace {

// mvs/src/fuse.rs:72-92: robust sparse bounding-box diagonal -> voxel cell
double voxel_cell(const double* xyz, uint64_t n, double voxel_rel) {
    double ext[3];
    for (int a = 0; a < 3; ++a) {
        std::vector<double> ax(n);
        for (uint64_t p = 0; p < n; ++p) ax[p] = xyz[3 * p + a];
        std::sort(ax.begin(), ax.end());
        size_t len = ax.size();
        size_t lo = std::min((size_t)((double)len * 0.02), len - 1);
        size_t hi = std::min((size_t)((double)len * 0.98), len - 1);
        ext[a] = ax[hi] - ax[lo];
    }
    double diag = std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]);
    return std::fmax(diag * voxel_rel, 1e-9);
}

// Fusion views of a scene; is_ref from ref_mask (every view when null).
int fuse_views(rcmvs_ctx* ctx, rcmvs_scene* sc, const int32_t* order_offsets, const int32_t* order,
               const std::vector<char>* ref_mask, std::vector<FuseView>& fv) {
    const int n = sc->n_views;
    for (int v = 0; v < n; ++v) {
        if (order_offsets[v] > order_offsets[v + 1] || order_offsets[v] < 0)
            return fail(ctx, RCMVS_E_ARG, "fusion order offsets must be non-decreasing");
        for (int32_t q = order_offsets[v]; q < order_offsets[v + 1]; ++q)
            if (!order || order[q] < 0 || order[q] >= n || !sc->has_depth[order[q]])
                return fail(ctx, RCMVS_E_ARG, "fusion order names a view without a depth map");
    }
    bool any = false;
    for (int v = 0; v < n; ++v) any |= sc->has_depth[v] != 0 && (!ref_mask || (*ref_mask)[v]);
    if (any && !sc->has_rgb) return fail(ctx, RCMVS_E_ARG, "fusion needs rgb for every view");
    fv.assign(n, FuseView{});
    for (int v = 0; v < n; ++v) {
        FuseView& F = fv[v];
        std::memset(&F, 0, sizeof(F));
        F.w = sc->views[v].w;
        F.h = sc->views[v].h;
        F.off = sc->views[v].off;
        F.has_depth = sc->has_depth[v];
        F.is_ref = ref_mask ? (*ref_mask)[v] : 1;
        F.order_begin = order_offsets[v];
        F.order_end = order_offsets[v + 1];
        const HostCam& c = sc->cams[v];
        F.f = c.f;
        F.cx = c.cx;
        F.cy = c.cy;
        F.k = c.k;
        std::memcpy(F.R, c.R, sizeof(F.R));
        std::memcpy(F.t, c.t, sizeof(F.t));
    }
    return RCMVS_OK;
}

// Library-allocated host copy of n points (device xyz / rgb) into out.
int take_points(rcmvs_ctx* ctx, const double* d_xyz, const uint8_t* d_rgb, uint64_t n, rcmvs_points* out) {
    out->xyz = (double*)std::malloc(24 * std::max<uint64_t>(n, 1));
    out->rgb = (uint8_t*)std::malloc(3 * std::max<uint64_t>(n, 1));
    if (!out->xyz || !out->rgb) {
        rcmvs_points_free(out);
        return fail(ctx, RCMVS_E_NOMEM, "host allocation of the point cloud failed");
    }
    out->n = n;
    if (n) {
        CK(cudaMemcpyAsync(out->xyz, d_xyz, 24 * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(out->rgb, d_rgb, 3 * n, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return RCMVS_OK;
}

}  // namespace

extern "C" {

int rcmvs_scene_fuse(rcmvs_ctx* ctx, rcmvs_scene* sc, const int32_t* order_offsets, const int32_t* order,
                     const double* sparse_xyz, uint64_t n_sparse, const rcmvs_options* opts, uint64_t* n_points_out) {
    if (!ctx || !sc || !order_offsets || !opts || !sparse_xyz || n_sparse == 0 || !n_points_out)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_fuse: bad argument (sparse cloud must be non-empty)");
    if (sc->ctx != ctx) return fail(ctx, RCMVS_E_ARG, "scene belongs to another context");
    const int n = sc->n_views;
    std::vector<FuseView> fv;
    int rc = fuse_views(ctx, sc, order_offsets, order, nullptr, fv);
    if (rc) return rc;
    const double cell = voxel_cell(sparse_xyz, n_sparse, opts->voxel_rel);
    CK(cudaSetDevice(ctx->device));
    FuseResult res{0, 0};
    std::string err;
    rc = fuse_device(sc->arena, fv.data(), n, order, order_offsets[n], sc->depth, sc->rgb, cell,
                     opts->min_consistent, opts->depth_diff, opts->reproj_px, &sc->d_pts_xyz, &sc->d_pts_rgb,
                     &sc->d_ply, &res, ctx->stream, &err, ctx->hook());
    if (rc) return fail(ctx, rc, err);
    sc->n_points = res.n_points;
    sc->n_candidates = res.n_candidates;
    *n_points_out = res.n_points;
    return RCMVS_OK;
}

int rcmvs_scene_fuse_candidates(rcmvs_ctx* ctx, rcmvs_scene* sc, const int32_t* order_offsets, const int32_t* order,
                                const int32_t* ref_views, int32_t n_ref, const rcmvs_options* opts,
                                rcmvs_points* out, uint64_t* per_view) {
    if (!ctx || !sc || !order_offsets || !opts || !out || n_ref < 0 || (n_ref > 0 && !ref_views))
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_fuse_candidates: bad argument");
    if (sc->ctx != ctx) return fail(ctx, RCMVS_E_ARG, "scene belongs to another context");
    out->n = 0;
    out->xyz = nullptr;
    out->rgb = nullptr;
    const int n = sc->n_views;
    std::vector<char> mask(n, 0);
    for (int i = 0; i < n_ref; ++i) {
        if (ref_views[i] < 0 || ref_views[i] >= n) return fail(ctx, RCMVS_E_ARG, "reference view out of range");
        mask[ref_views[i]] = 1;
    }
    std::vector<FuseView> fv;
    int rc = fuse_views(ctx, sc, order_offsets, order, &mask, fv);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    std::string err;
    const uint32_t* cand = nullptr;
    const double* pts = nullptr;
    uint32_t n_cand = 0;
    rc = fuse_candidates_device(sc->arena, fv.data(), n, order, order_offsets[n], sc->depth, opts->min_consistent,
                                opts->depth_diff, opts->reproj_px, &cand, &n_cand, &pts, ctx->stream, &err,
                                ctx->hook());
    if (rc) return fail(ctx, rc, err);
    double* gx = nullptr;
    uint8_t* gc = nullptr;
    if (n_cand > 0) {
        rc = fuse_gather_device(sc->arena, cand, n_cand, pts, sc->rgb, &gx, &gc, ctx->stream, &err);
        if (rc) return fail(ctx, rc, err);
    }
    if (per_view) {
        // candidates are ascending global pixel indices; views are laid out
        // in order, so each view's candidates form one run
        std::vector<uint32_t> idx(n_cand);
        if (n_cand) CK(cudaMemcpyAsync(idx.data(), cand, 4 * (size_t)n_cand, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        size_t c = 0;
        for (int v = 0; v < n; ++v) {
            const uint64_t end = (uint64_t)sc->views[v].off + (uint64_t)sc->views[v].w * sc->views[v].h;
            uint64_t k = 0;
            while (c < idx.size() && idx[c] < end) {
                ++c;
                ++k;
            }
            per_view[v] = k;
        }
    }
    return take_points(ctx, gx, gc, n_cand, out);
}

int rcmvs_scene_fuse_candidates_device(rcmvs_ctx* ctx, rcmvs_scene* sc, const int32_t* order_offsets,
                                       const int32_t* order, const int32_t* ref_views, int32_t n_ref,
                                       const rcmvs_options* opts, uint64_t* n_out, uint64_t* per_view) {
    if (!ctx || !sc || !order_offsets || !opts || !n_out || n_ref < 0 || (n_ref > 0 && !ref_views))
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_fuse_candidates_device: bad argument");
    if (sc->ctx != ctx) return fail(ctx, RCMVS_E_ARG, "scene belongs to another context");
    *n_out = 0;
    sc->n_kept = 0;
    sc->d_kept_xyz = nullptr;
    sc->d_kept_rgb = nullptr;
    const int n = sc->n_views;
    std::vector<char> mask(n, 0);
    for (int i = 0; i < n_ref; ++i) {
        if (ref_views[i] < 0 || ref_views[i] >= n) return fail(ctx, RCMVS_E_ARG, "reference view out of range");
        mask[ref_views[i]] = 1;
    }
    std::vector<FuseView> fv;
    int rc = fuse_views(ctx, sc, order_offsets, order, &mask, fv);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    std::string err;
    const uint32_t* cand = nullptr;
    const double* pts = nullptr;
    uint32_t n_cand = 0;
    rc = fuse_candidates_device(sc->arena, fv.data(), n, order, order_offsets[n], sc->depth, opts->min_consistent,
                                opts->depth_diff, opts->reproj_px, &cand, &n_cand, &pts, ctx->stream, &err,
                                ctx->hook());
    if (rc) return fail(ctx, rc, err);
    double* gx = nullptr;
    uint8_t* gc = nullptr;
    rc = fuse_gather_device(sc->arena, cand, n_cand, pts, sc->rgb, &gx, &gc, ctx->stream, &err);
    if (rc) return fail(ctx, rc, err);
    if (per_view) {
        std::vector<uint32_t> idx(n_cand);
        if (n_cand) CK(cudaMemcpyAsync(idx.data(), cand, 4 * (size_t)n_cand, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        size_t c = 0;
        for (int v = 0; v < n; ++v) {
            const uint64_t end = (uint64_t)sc->views[v].off + (uint64_t)sc->views[v].w * sc->views[v].h;
            uint64_t k = 0;
            while (c < idx.size() && idx[c] < end) {
                ++c;
                ++k;
            }
            per_view[v] = k;
        }
    }
    sc->n_kept = n_cand;
    sc->d_kept_xyz = gx;
    sc->d_kept_rgb = gc;
    *n_out = n_cand;
    return RCMVS_OK;
}

int rcmvs_scene_candidates_to_device(rcmvs_ctx* ctx, rcmvs_scene* sc, double* xyz_dev, uint8_t* rgb_dev) {
    if (!ctx || !sc || (sc->n_kept > 0 && (!xyz_dev || !rgb_dev)))
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_candidates_to_device: bad argument");
    if (sc->n_kept == 0) return RCMVS_OK;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(xyz_dev, sc->d_kept_xyz, 24 * sc->n_kept, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(rgb_dev, sc->d_kept_rgb, 3 * sc->n_kept, cudaMemcpyDeviceToDevice, ctx->stream));
    return RCMVS_OK;
}

int rcmvs_scene_fuse_reduce_device(rcmvs_ctx* ctx, rcmvs_scene* sc, const double* xyz_dev, const uint8_t* rgb_dev,
                                   uint64_t n, const double* sparse_xyz, uint64_t n_sparse,
                                   const rcmvs_options* opts, uint64_t* n_points_out) {
    if (!ctx || !sc || (n > 0 && (!xyz_dev || !rgb_dev)) || !sparse_xyz || n_sparse == 0 || !opts || !n_points_out)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_fuse_reduce_device: bad argument (sparse cloud must be non-empty)");
    if (sc->ctx != ctx) return fail(ctx, RCMVS_E_ARG, "scene belongs to another context");
    CK(cudaSetDevice(ctx->device));
    const double cell = voxel_cell(sparse_xyz, n_sparse, opts->voxel_rel);
    std::string err;
    uint64_t np = 0;
    int rc = fuse_reduce_devptr(sc->arena, xyz_dev, rgb_dev, n, cell, &sc->d_pts_xyz, &sc->d_pts_rgb, &sc->d_ply, &np,
                                ctx->stream, &err, ctx->hook());
    if (rc) return fail(ctx, rc, err);
    sc->n_points = np;
    sc->n_candidates = n;
    *n_points_out = np;
    return RCMVS_OK;
}

int rcmvs_fuse_reduce(rcmvs_ctx* ctx, const double* xyz, const uint8_t* rgb, uint64_t n, const double* sparse_xyz,
                      uint64_t n_sparse, const rcmvs_options* opts, rcmvs_points* out) {
    if (!ctx || (n > 0 && (!xyz || !rgb)) || !sparse_xyz || n_sparse == 0 || !opts || !out)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_fuse_reduce: bad argument (sparse cloud must be non-empty)");
    out->n = 0;
    out->xyz = nullptr;
    out->rgb = nullptr;
    CK(cudaSetDevice(ctx->device));
    const double cell = voxel_cell(sparse_xyz, n_sparse, opts->voxel_rel);
    double* dx = nullptr;
    uint8_t *dc = nullptr, *dp = nullptr;
    uint64_t np = 0;
    std::string err;
    int rc = fuse_reduce_host(ctx->arena, xyz, rgb, n, cell, &dx, &dc, &dp, &np, ctx->stream, &err, ctx->hook());
    if (rc) return fail(ctx, rc, err);
    return take_points(ctx, dx, dc, np, out);
}

int rcmvs_scene_get_points(rcmvs_ctx* ctx, rcmvs_scene* sc, double* xyz, uint8_t* rgb, uint8_t* ply_body) {
    if (!ctx || !sc) return fail(ctx, RCMVS_E_ARG, "rcmvs_scene_get_points: bad argument");
    if (sc->n_points == 0) return RCMVS_OK;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t n = sc->n_points;
    if (xyz) CK(cudaMemcpyAsync(xyz, sc->d_pts_xyz, 24 * n, cudaMemcpyDeviceToHost, st));
    if (rgb) CK(cudaMemcpyAsync(rgb, sc->d_pts_rgb, 3 * n, cudaMemcpyDeviceToHost, st));
    if (ply_body) CK(cudaMemcpyAsync(ply_body, sc->d_ply, 15 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return RCMVS_OK;
}

// ================================================================ host API
int rcmvs_census(rcmvs_ctx* ctx, const uint8_t* gray, int32_t w, int32_t h, uint64_t* census_out) {
    if (!ctx || !gray || !census_out || w <= 0 || h <= 0) return fail(ctx, RCMVS_E_ARG, "rcmvs_census: bad argument");
    rcmvs_view v;
    std::memset(&v, 0, sizeof(v));
    v.w = w;
    v.h = h;
    v.f = 1.0;
    v.R[0] = v.R[4] = v.R[8] = 1.0;
    v.gray = gray;
    rcmvs_scene* sc = nullptr;
    int rc = rcmvs_scene_create(ctx, &v, 1, &sc);
    if (rc) return rc;
    rc = rcmvs_scene_get_census(ctx, sc, 0, census_out);
    rcmvs_scene_destroy(sc);
    return rc;
}

// Builds a scene of the views jobs touch; remap[] maps caller view -> scene view.
static int sub_scene(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, const rcmvs_job* jobs, int32_t n_jobs,
                     const rcmvs_options* opts, std::vector<int>& remap, rcmvs_scene** out) {
    remap.assign(n_views, -1);
    std::vector<rcmvs_view> sub;
    auto use = [&](int v) {
        if (remap[v] < 0) {
            remap[v] = (int)sub.size();
            sub.push_back(views[v]);
        }
    };
    for (int j = 0; j < n_jobs; ++j) {
        use(jobs[j].ref_idx);
        for (int s = 0; s < jobs[j].n_src; ++s) use(jobs[j].srcs[s]);
    }
    for (size_t i = 0; i < sub.size(); ++i) {
        int rc = check_view(ctx, sub[i], (int)i, nullptr);
        if (rc) return rc;
    }
    (void)opts;
    return rcmvs_scene_create(ctx, sub.data(), (int32_t)sub.size(), out);
}

int rcmvs_estimate_depth_batch(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, const rcmvs_job* jobs,
                               int32_t n_jobs, const rcmvs_options* opts, const rcmvs_depth_out* outs) {
    if (!ctx || !views || n_views <= 0 || !opts || (n_jobs > 0 && !outs))
        return fail(ctx, RCMVS_E_ARG, "rcmvs_estimate_depth_batch: bad argument");
    int rc = validate_jobs(ctx, n_views, jobs, n_jobs);
    if (rc) return rc;
    for (int j = 0; j < n_jobs; ++j)
        if (!outs[j].depth || !outs[j].cost) return fail(ctx, RCMVS_E_ARG, "null depth/cost output");
    if (n_jobs == 0) return RCMVS_OK;
    std::vector<int> remap;
    rcmvs_scene* sc = nullptr;
    rc = sub_scene(ctx, views, n_views, jobs, n_jobs, opts, remap, &sc);
    if (rc) return rc;
    std::vector<rcmvs_job> sj(jobs, jobs + n_jobs);
    std::vector<std::vector<int32_t>> ss(n_jobs);
    for (int j = 0; j < n_jobs; ++j) {
        for (int s = 0; s < jobs[j].n_src; ++s) ss[j].push_back(remap[jobs[j].srcs[s]]);
        sj[j].ref_idx = remap[jobs[j].ref_idx];
        sj[j].srcs = ss[j].data();
    }
    rc = rcmvs_scene_estimate_depth(ctx, sc, sj.data(), n_jobs, opts);
    for (int j = 0; j < n_jobs && rc == RCMVS_OK; ++j)
        rc = rcmvs_scene_get_depth(ctx, sc, sj[j].ref_idx, outs[j].depth, outs[j].cost, outs[j].normal);
    rcmvs_scene_destroy(sc);
    return rc;
}

int rcmvs_estimate_depth(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                         const int32_t* srcs, int32_t n_src, double zmin, double zmax, const rcmvs_options* opts,
                         float* depth_out, float* cost_out, float* normal_out) {
    rcmvs_job j{ref_idx, n_src, srcs, zmin, zmax};
    rcmvs_depth_out o{depth_out, cost_out, normal_out};
    return rcmvs_estimate_depth_batch(ctx, views, n_views, &j, 1, opts, &o);
}

int rcmvs_plane_cost_field(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                           const int32_t* srcs, int32_t n_src, const float* planes, const float* hints,
                           float* cost_out, int32_t* hsum_out) {
    if (!ctx || !views || !planes || !hints || !cost_out)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_plane_cost_field: bad argument");
    rcmvs_job job{ref_idx, n_src, srcs, 1.0, 2.0};
    int rc = validate_jobs(ctx, n_views, &job, 1);
    if (rc) return rc;
    std::vector<int> remap;
    rcmvs_scene* sc = nullptr;
    rc = sub_scene(ctx, views, n_views, &job, 1, nullptr, remap, &sc);
    if (rc) return rc;
    const TileShape ts{16, 16};
    std::vector<int32_t> ss;
    for (int s = 0; s < n_src; ++s) ss.push_back(remap[srcs[s]]);
    DevJob hj;
    fill_job(sc, remap[ref_idx], ss.data(), n_src, 1.0, 2.0, ts, hj);
    hj.tile_base = 0;
    int32_t start[2] = {0, hj.tiles};
    const size_t n = (size_t)views[ref_idx].w * views[ref_idx].h;
    void *pj, *ps, *ppl, *ph, *pc, *phs;
    cudaStream_t st = ctx->stream;
    auto body = [&]() -> int {
        CK(ctx->arena.get(S_JOBS, sizeof(DevJob), &pj));
        CK(ctx->arena.get(S_JOBSTART, sizeof(start), &ps));
        CK(ctx->arena.get(S_FIELD_PL, 16 * n, &ppl));
        CK(ctx->arena.get(S_FIELD_H, 4 * n, &ph));
        CK(ctx->arena.get(S_FIELD_C, 4 * n, &pc));
        CK(ctx->arena.get(S_FIELD_HS, 4 * n, &phs));
        CK(cudaMemcpyAsync(pj, &hj, sizeof(DevJob), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ps, start, sizeof(start), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ppl, planes, 16 * n, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ph, hints, 4 * n, cudaMemcpyHostToDevice, st));
        const LaunchGeom g{ts.tw * ts.th, stereo_smem_bytes(ts), hj.tiles, nullptr};
        CK(launch_cost_field((const DevJob*)pj, (const int32_t*)ps, g, sc->census, sc->rays,
                             (const float4*)ppl, (const float*)ph, (float*)pc, (int32_t*)phs, st));
        CK(cudaMemcpyAsync(cost_out, pc, 4 * n, cudaMemcpyDeviceToHost, st));
        if (hsum_out) CK(cudaMemcpyAsync(hsum_out, phs, 4 * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return RCMVS_OK;
    };
    rc = body();
    rcmvs_scene_destroy(sc);
    return rc;
}

int rcmvs_selftest_f2i(rcmvs_ctx* ctx, const float* in, int32_t n, int32_t* out) {
    if (!ctx || !in || !out || n <= 0) return fail(ctx, RCMVS_E_ARG, "rcmvs_selftest_f2i: bad argument");
    CK(cudaSetDevice(ctx->device));
    void *pi, *po;
    CK(ctx->arena.get(S_CGRAY, 4 * (size_t)n, &pi));
    CK(ctx->arena.get(S_F2I, 4 * (size_t)n, &po));
    CK(cudaMemcpyAsync(pi, in, 4 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_f2i((const float*)pi, n, (int32_t*)po, ctx->stream));
    CK(cudaMemcpyAsync(out, po, 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return RCMVS_OK;
}

int rcmvs_fuse_depth_maps(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, const float* const* depth_maps,
                          const int32_t* order_offsets, const int32_t* order, const double* sparse_xyz,
                          uint64_t n_sparse, const rcmvs_options* opts, rcmvs_points* out) {
    if (!ctx || !views || n_views <= 0 || !depth_maps || !order_offsets || !opts || !out)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_fuse_depth_maps: bad argument");
    out->n = 0;
    out->xyz = nullptr;
    out->rgb = nullptr;
    rcmvs_scene* sc = nullptr;
    int rc = rcmvs_scene_create(ctx, views, n_views, &sc);
    if (rc) return rc;
    auto body = [&]() -> int {
        cudaStream_t st = ctx->stream;
        for (int v = 0; v < n_views; ++v) {
            if (!depth_maps[v]) continue;
            const DevView& V = sc->views[v];
            CK(cudaMemcpyAsync(sc->depth + V.off, depth_maps[v], 4 * (size_t)V.w * V.h, cudaMemcpyHostToDevice, st));
            sc->has_depth[v] = 1;
        }
        uint64_t np = 0;
        int r = rcmvs_scene_fuse(ctx, sc, order_offsets, order, sparse_xyz, n_sparse, opts, &np);
        if (r) return r;
        out->xyz = (double*)std::malloc(24 * std::max<uint64_t>(np, 1));
        out->rgb = (uint8_t*)std::malloc(3 * std::max<uint64_t>(np, 1));
        if (!out->xyz || !out->rgb) {
            rcmvs_points_free(out);
            return fail(ctx, RCMVS_E_NOMEM, "host allocation of the point cloud failed");
        }
        out->n = np;
        return rcmvs_scene_get_points(ctx, sc, out->xyz, out->rgb, nullptr);
    };
    rc = body();
    rcmvs_scene_destroy(sc);
    return rc;
}

int rcmvs_fuse_candidates(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, const float* const* depth_maps,
                          const int32_t* order_offsets, const int32_t* order, const int32_t* ref_views,
                          int32_t n_ref, const rcmvs_options* opts, rcmvs_points* out, uint64_t* per_view) {
    if (!ctx || !views || n_views <= 0 || !depth_maps || !order_offsets || !opts || !out)
        return fail(ctx, RCMVS_E_ARG, "rcmvs_fuse_candidates: bad argument");
    out->n = 0;
    out->xyz = nullptr;
    out->rgb = nullptr;
    rcmvs_scene* sc = nullptr;
    int rc = rcmvs_scene_create(ctx, views, n_views, &sc);
    if (rc) return rc;
    auto body = [&]() -> int {
        for (int v = 0; v < n_views; ++v) {
            if (!depth_maps[v]) continue;
            const DevView& V = sc->views[v];
            CK(cudaMemcpyAsync(sc->depth + V.off, depth_maps[v], 4 * (size_t)V.w * V.h, cudaMemcpyHostToDevice,
                               ctx->stream));
            sc->has_depth[v] = 1;
        }
        return rcmvs_scene_fuse_candidates(ctx, sc, order_offsets, order, ref_views, n_ref, opts, out, per_view);
    };
    rc = body();
    rcmvs_scene_destroy(sc);
    return rc;
}

// mvs/src/fuse.rs:222-239
// mvs/src/lib.rs:434-485: the decimated copy for web viewers.  Centroid as
// sequential f64 sums, distances to it, the robust radius med + 6 *
// max(|p95 - med|, max(med, 1e-9) / 2) from the sorted distances, then every
// stride-th kept point (stride = ceil(kept / cap)), in the cloud's order.
static int write_web_json(const std::string& path, const double* xyz, const uint8_t* rgb, uint64_t n,
                          uint64_t cap) {
    if (n == 0) return RCMVS_OK;  // the reference writes no file for an empty cloud
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (uint64_t i = 0; i < n; ++i) sx += xyz[3 * i];
    for (uint64_t i = 0; i < n; ++i) sy += xyz[3 * i + 1];
    for (uint64_t i = 0; i < n; ++i) sz += xyz[3 * i + 2];
    const double cx = sx / (double)n, cy = sy / (double)n, cz = sz / (double)n;
    std::vector<double> d(n);
    for (uint64_t i = 0; i < n; ++i) {
        const double dx = xyz[3 * i] - cx, dy = xyz[3 * i + 1] - cy, dz = xyz[3 * i + 2] - cz;
        d[i] = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    std::vector<double> sd(d);
    std::sort(sd.begin(), sd.end());
    const double med = sd[n / 2];
    const double p95 = sd[std::min<uint64_t>((uint64_t)((double)n * 0.95), n - 1)];
    const double r_keep = med + 6.0 * std::max(std::fabs(p95 - med), std::max(med, 1e-9) * 0.5);
    std::vector<uint64_t> kept;
    for (uint64_t i = 0; i < n; ++i)
        if (d[i] <= r_keep) kept.push_back(i);
    const uint64_t stride = std::max<uint64_t>((kept.size() + cap - 1) / cap, 1);
    std::vector<uint64_t> web;
    for (uint64_t k = 0; k < kept.size(); k += stride) web.push_back(kept[k]);
    std::string out = "{\"n\":" + std::to_string(web.size()) + ",\"pos\":[";
    char tmp[128];
    for (size_t k = 0; k < web.size(); ++k) {
        const uint64_t i = web[k];
        std::snprintf(tmp, sizeof(tmp), "%s[%.4f,%.4f,%.4f]", k ? "," : "", xyz[3 * i], xyz[3 * i + 1],
                      xyz[3 * i + 2]);
        out += tmp;
    }
    out += "],\"col\":[";
    for (size_t k = 0; k < web.size(); ++k) {
        const uint64_t i = web[k];
        std::snprintf(tmp, sizeof(tmp), "%s[%u, %u,%u]", k ? "," : "", rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
        out += tmp;
    }
    out += "]}";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return RCMVS_E_IO;
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return (std::fclose(f) == 0 && ok) ? RCMVS_OK : RCMVS_E_IO;
}

int rcmvs_write_dense_outputs(const char* dense_dir, const double* xyz, const uint8_t* rgb, uint64_t n,
                              const rcmvs_stats* stats, uint64_t web_cap) {
    if (!dense_dir || (n > 0 && (!xyz || !rgb))) return RCMVS_E_ARG;
    const std::string dir(dense_dir);
    int rc = rcmvs_write_ply_binary((dir + "/dense.ply").c_str(), xyz, rgb, n);
    if (rc) return rc;
    rc = write_web_json(dir + "/dense_web.json", xyz, rgb, n, web_cap ? web_cap : 400000);
    if (rc) return rc;
    if (stats) {  // mvs/src/lib.rs:497-501
        FILE* f = std::fopen((dir + "/mvs_stats.json").c_str(), "wb");
        if (!f) return RCMVS_E_IO;
        std::fprintf(f,
                     "{\"views\": %llu, \"views_with_depth\": %llu, \"dense_points\": %llu, \"stereo_s\": %.1f, "
                     "\"fuse_s\": %.1f, \"elapsed_s\": %.1f}",
                     (unsigned long long)stats->views, (unsigned long long)stats->views_with_depth,
                     (unsigned long long)stats->dense_points, (double)stats->stereo_s, (double)stats->fuse_s,
                     (double)stats->elapsed_s);
        if (std::fclose(f) != 0) return RCMVS_E_IO;
    }
    return RCMVS_OK;
}

int rcmvs_write_ply_binary(const char* path, const double* xyz, const uint8_t* rgb, uint64_t n) {
    if (!path || (n > 0 && (!xyz || !rgb))) return RCMVS_E_ARG;
    FILE* f = std::fopen(path, "wb");
    if (!f) return RCMVS_E_IO;
    std::fprintf(f,
                 "ply\nformat binary_little_endian 1.0\ncomment rustcolmap dense MVS fusion\n"
                 "element vertex %llu\nproperty float x\nproperty float y\nproperty float z\n"
                 "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n",
                 (unsigned long long)n);
    std::vector<uint8_t> buf;
    buf.reserve(15 * std::min<uint64_t>(n, 1 << 16));
    for (uint64_t i = 0; i < n; ++i) {
        float p[3] = {(float)xyz[3 * i], (float)xyz[3 * i + 1], (float)xyz[3 * i + 2]};
        const uint8_t* b = reinterpret_cast<const uint8_t*>(p);  // x86-64 / aarch64: little-endian
        buf.insert(buf.end(), b, b + 12);
        buf.insert(buf.end(), rgb + 3 * i, rgb + 3 * i + 3);
        if (buf.size() >= 15u * (1u << 16)) {
            if (std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) {
                std::fclose(f);
                return RCMVS_E_IO;
            }
            buf.clear();
        }
    }
    if (!buf.empty() && std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) {
        std::fclose(f);
        return RCMVS_E_IO;
    }
    return std::fclose(f) == 0 ? RCMVS_OK : RCMVS_E_IO;
}

}  // extern "C"

// ================================================================ plan
namespace {
// mvs/src/lib.rs:245-251
double percentile(const std::vector<double>& s, double q) {
    if (s.empty()) return 0.0;
    double idx = std::round(((double)s.size() - 1.0) * q);
    idx = std::min(std::max(idx, 0.0), (double)s.size() - 1.0);
    return s[(size_t)idx];
}

// The same on an unsorted sample: the element a sort would put at that
// index, found by selection (same value, linear time; reorders s).
double percentile_select(std::vector<double>& s, double q) {
    if (s.empty()) return 0.0;
    double idx = std::round(((double)s.size() - 1.0) * q);
    idx = std::min(std::max(idx, 0.0), (double)s.size() - 1.0);
    auto it = s.begin() + (std::ptrdiff_t)idx;
    std::nth_element(s.begin(), it, s.end());
    return *it;
}

// Runs f(t, begin, end) on nt threads over [0, n) in contiguous chunks.
template <class F>
void par_chunks(int64_t n, int nt, F&& f) {
    nt = (int)std::max<int64_t>(1, std::min<int64_t>(nt, n));
    if (nt == 1) {
        f(0, (int64_t)0, n);
        return;
    }
    std::vector<std::thread> ts;
    for (int t = 0; t < nt; ++t)
        ts.emplace_back([&, t] { f(t, n * t / nt, n * (t + 1) / nt); });
    for (auto& th : ts) th.join();
}

int plan_threads() {
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::min(16u, std::max(1u, hc));
}
}  // namespace

extern "C" {

// Host glue of run_mvs (mvs/src/lib.rs:224-282, :303-342, :398-418).  The
// count sorts keep ascending view index among equal counts; the reference's
// unstable sort agrees whenever a list has <= 20 entries (insertion sort) or
// no ties.
int rcmvs_plan(const rcmvs_sparse* sp, const rcmvs_view* views, int32_t n_views, const rcmvs_options* opts,
               int32_t* src_offsets, int32_t* srcs, double* zrange, int32_t* fuse_offsets, int32_t* fuse_order) {
    if (!sp || !views || n_views <= 0 || !opts || !src_offsets || !srcs || !zrange || !fuse_offsets || !fuse_order)
        return RCMVS_E_ARG;
    if (sp->n_points < 8 || !sp->xyz || !sp->track_offsets || (sp->track_offsets[sp->n_points] > 0 && !sp->track_views))
        return RCMVS_E_ARG;  // lib.rs:310-315
    const int n = n_views;
    std::vector<double> global(sp->n_points);
    for (uint64_t p = 0; p < sp->n_points; ++p) {
        const double* x = sp->xyz + 3 * p;
        global[p] = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    }
    std::sort(global.begin(), global.end());
    // co-visibility counts and the points each view sees (lib.rs:224-243):
    // integer counts, summed over threads that each take a range of points
    // with their own count matrix (at most 256 MB of them)
    const int nt = (int)std::max<int64_t>(
        1, std::min<int64_t>(plan_threads(), (int64_t(64) << 20) / std::max<int64_t>(1, (int64_t)n * n)));
    std::vector<std::vector<uint32_t>> covt(nt, std::vector<uint32_t>((size_t)n * n, 0));
    std::vector<std::vector<std::vector<uint64_t>>> seen_t(nt, std::vector<std::vector<uint64_t>>(n));
    par_chunks((int64_t)sp->n_points, nt, [&](int t, int64_t p0, int64_t p1) {
        std::vector<int> ids;
        std::vector<uint32_t>& cv = covt[t];
        for (int64_t p = p0; p < p1; ++p) {
            ids.clear();
            for (uint64_t q = sp->track_offsets[p]; q < sp->track_offsets[p + 1]; ++q) {
                int v = sp->track_views[q];
                if (v >= 0 && v < n) ids.push_back(v);
            }
            std::sort(ids.begin(), ids.end());
            ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
            for (int a : ids) {
                seen_t[t][a].push_back((uint64_t)p);
                for (int b : ids)
                    if (a != b) cv[(size_t)a * n + b]++;
            }
        }
    });
    std::vector<uint32_t>& cov = covt[0];
    for (int t = 1; t < nt; ++t)
        for (size_t e = 0; e < cov.size(); ++e) cov[e] += covt[t][e];
    std::vector<std::vector<int>> sources(n);
    std::vector<char> has(n, 0);
    int off = 0;
    for (int i = 0; i < n; ++i) {
        std::vector<std::pair<uint32_t, int>> o;
        for (int j = 0; j < n; ++j)
            if (cov[(size_t)i * n + j] >= 10) o.push_back({cov[(size_t)i * n + j], j});
        std::stable_sort(o.begin(), o.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        src_offsets[i] = off;
        for (size_t q = 0; q < o.size() && q < opts->num_sources; ++q) {
            sources[i].push_back(o[q].second);
            srcs[off++] = o[q].second;
        }
        has[i] = !sources[i].empty();
    }
    src_offsets[n] = off;
    // depth_range_for (lib.rs:253-282), views in parallel; the percentiles
    // are order statistics, so selection gives the sorted list's values
    par_chunks(n, plan_threads(), [&](int, int64_t i0, int64_t i1) {
        std::vector<double> ds;
        for (int64_t i = i0; i < i1; ++i) {
            const rcmvs_view& v = views[i];
            ds.clear();
            for (int t = 0; t < nt; ++t)
                for (uint64_t p : seen_t[t][i]) {
                    const double* x = sp->xyz + 3 * p;
                    double z = (v.R[6] * x[0] + v.R[7] * x[1] + v.R[8] * x[2]) + v.t[2];
                    if (z > 1e-6) ds.push_back(z);
                }
            double lo = 0.0, hi = 0.0;
            if (ds.size() >= 8) {
                lo = percentile_select(ds, 0.02);
                hi = percentile_select(ds, 0.98);
            } else if (global.size() >= 8) {
                lo = percentile(global, 0.02);
                hi = percentile(global, 0.98);
            }
            if (hi <= lo * 1.05 || lo <= 0.0) {
                zrange[2 * i] = std::fmax(percentile(global, 0.01) * 0.7, 1e-3);
                zrange[2 * i + 1] = percentile(global, 0.99) * 1.4;
            } else {
                zrange[2 * i] = lo * 0.8;
                zrange[2 * i + 1] = hi * 1.25;
            }
        }
    });
    off = 0;
    for (int i = 0; i < n; ++i) {  // fusion order, sources first (lib.rs:398-418)
        std::vector<std::pair<uint32_t, int>> o;
        for (int j = 0; j < n; ++j)
            if (cov[(size_t)i * n + j] >= 10 && has[j]) o.push_back({cov[(size_t)i * n + j], j});
        std::stable_sort(o.begin(), o.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        const auto& s = sources[i];
        auto rank = [&](int j) -> size_t {
            auto it = std::find(s.begin(), s.end(), j);
            return it == s.end() ? SIZE_MAX : (size_t)(it - s.begin());
        };
        std::stable_sort(o.begin(), o.end(), [&](const auto& a, const auto& b) { return rank(a.second) < rank(b.second); });
        fuse_offsets[i] = off;
        for (auto& c : o) fuse_order[off++] = c.second;
    }
    fuse_offsets[n] = off;
    return RCMVS_OK;
}

}  // extern "C"

// run_mvs with either the reference's plane-sweep init (net == NULL) or the
// learned init of rcmvs_scene_estimate_depth_learned.
static int run_mvs_impl(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, const rcmvs_sparse* sparse,
                        const rcmvs_options* opts, const rcmvs_depth_out* depth_outs, rcmvs_points* out,
                        rcmvs_stats* stats, rcmvs_net* net, float conf_thr, int32_t n_local, float span) {
    if (!ctx || !views || !sparse || !opts || !out) return fail(ctx, RCMVS_E_ARG, "rcmvs_run_mvs: bad argument");
    out->n = 0;
    out->xyz = nullptr;
    out->rgb = nullptr;
    if (n_views < 2) return fail(ctx, RCMVS_E_ARG, "need at least 2 registered views for MVS");  // lib.rs:175-177
    if (sparse->n_points < 8)
        return fail(ctx, RCMVS_E_ARG, "sparse reconstruction too small for MVS (need >= 8 points)");
    for (int i = 0; i < n_views; ++i) {
        int rc = check_view(ctx, views[i], i, opts);
        if (rc) return rc;
        if (!views[i].rgb) return fail(ctx, RCMVS_E_ARG, "run_mvs needs rgb for every view");
    }
    cudaEvent_t e0, e1, e2, e3;
    CK(cudaSetDevice(ctx->device));
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventCreate(&e2));
    CK(cudaEventCreate(&e3));
    const int n = n_views;
    rcmvs_scene* sc = nullptr;
    CK(cudaEventRecord(e0, ctx->stream));
    // the RGB uploads (three quarters of the input bytes) overlap the
    // stereo: only fusion reads them
    if (!ctx->upload) CK(cudaStreamCreateWithFlags(&ctx->upload, cudaStreamNonBlocking));
    cudaEvent_t rgb_done;
    CK(cudaEventCreateWithFlags(&rgb_done, cudaEventDisableTiming));
    int rc = scene_create(ctx, views, n, &sc, ctx->upload, rgb_done);
    if (rc) {
        cudaEventDestroy(rgb_done);
        return rc;
    }
    // the plan glue runs on the host while the uploads and the census run
    std::vector<int32_t> so(n + 1), ss((size_t)n * std::max<uint32_t>(opts->num_sources, 1u)), fo(n + 1),
        ff((size_t)n * n);
    std::vector<double> zr(2 * n);
    std::vector<rcmvs_job> jobs;
    rc = rcmvs_plan(sparse, views, n, opts, so.data(), ss.data(), zr.data(), fo.data(), ff.data());
    if (rc) {
        cudaEventSynchronize(rgb_done);
        cudaEventDestroy(rgb_done);
        rcmvs_scene_destroy(sc);
        return fail(ctx, rc, "plan failed");
    }
    for (int i = 0; i < n; ++i)
        if (so[i + 1] > so[i]) jobs.push_back(rcmvs_job{i, so[i + 1] - so[i], ss.data() + so[i], zr[2 * i], zr[2 * i + 1]});
    auto body = [&]() -> int {
        CK(cudaEventRecord(e1, ctx->stream));
        int r = net ? rcmvs_scene_estimate_depth_learned(ctx, sc, jobs.data(), (int32_t)jobs.size(), opts, net,
                                                         conf_thr, n_local, span, nullptr)
                    : rcmvs_scene_estimate_depth(ctx, sc, jobs.data(), (int32_t)jobs.size(), opts);
        if (r) return r;
        CK(cudaEventRecord(e2, ctx->stream));
        CK(cudaStreamWaitEvent(ctx->stream, rgb_done, 0));
        uint64_t np = 0;
        r = rcmvs_scene_fuse(ctx, sc, fo.data(), ff.data(), sparse->xyz, sparse->n_points, opts, &np);
        if (r) return r;
        out->xyz = (double*)std::malloc(24 * std::max<uint64_t>(np, 1));
        out->rgb = (uint8_t*)std::malloc(3 * std::max<uint64_t>(np, 1));
        if (!out->xyz || !out->rgb) {
            rcmvs_points_free(out);
            return fail(ctx, RCMVS_E_NOMEM, "host allocation of the point cloud failed");
        }
        out->n = np;
        r = rcmvs_scene_get_points(ctx, sc, out->xyz, out->rgb, nullptr);
        if (r) return r;
        CK(cudaEventRecord(e3, ctx->stream));
        std::vector<float> zero;
        for (int i = 0; i < n && depth_outs; ++i) {
            const rcmvs_depth_out& d = depth_outs[i];
            if (sc->has_depth[i]) {
                r = rcmvs_scene_get_depth(ctx, sc, i, d.depth, d.cost, d.normal);
                if (r) return r;
            } else {
                const size_t np2 = (size_t)views[i].w * views[i].h;
                if (d.depth) std::fill(d.depth, d.depth + np2, 0.0f);
                if (d.cost) std::fill(d.cost, d.cost + np2, 1.0f);
                if (d.normal) std::fill(d.normal, d.normal + 3 * np2, 0.0f);
            }
        }
        CK(cudaStreamSynchronize(ctx->stream));
        if (stats) {
            float t_all = 0, t_st = 0, t_fu = 0;
            cudaEventElapsedTime(&t_all, e0, e3);
            cudaEventElapsedTime(&t_st, e1, e2);
            cudaEventElapsedTime(&t_fu, e2, e3);
            stats->views = n;
            stats->views_with_depth = jobs.size();
            stats->dense_points = np;
            stats->fusion_candidates = sc->n_candidates;
            stats->elapsed_s = t_all * 1e-3f;
            stats->stereo_s = t_st * 1e-3f;
            stats->fuse_s = t_fu * 1e-3f;
        }
        return RCMVS_OK;
    };
    rc = body();
    cudaEventSynchronize(rgb_done);  // the uploads read the caller's views and write the scene
    cudaEventDestroy(rgb_done);
    rcmvs_scene_destroy(sc);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    cudaEventDestroy(e3);
    if (rc) rcmvs_points_free(out);
    return rc;
}

extern "C" {

int rcmvs_run_mvs(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, const rcmvs_sparse* sparse,
                  const rcmvs_options* opts, const rcmvs_depth_out* depth_outs, rcmvs_points* out, rcmvs_stats* stats) {
    return run_mvs_impl(ctx, views, n_views, sparse, opts, depth_outs, out, stats, nullptr, 0.f, 1, 0.f);
}

int rcmvs_run_mvs_learned(rcmvs_ctx* ctx, const rcmvs_view* views, int32_t n_views, const rcmvs_sparse* sparse,
                          const rcmvs_options* opts, rcmvs_net* net, float conf_thr, int32_t n_local, float span,
                          const rcmvs_depth_out* depth_outs, rcmvs_points* out, rcmvs_stats* stats) {
    if (!net) return fail(ctx, RCMVS_E_ARG, "rcmvs_run_mvs_learned: null network");
    return run_mvs_impl(ctx, views, n_views, sparse, opts, depth_outs, out, stats, net, conf_thr, n_local, span);
}

}  // extern "C"
