// schedule.cu — host side of one stereo batch: all reference views of a
// scene (the per-view `estimate_depth` calls of mvs/src/lib.rs:345-370) in
// one launch per step.
//
//   * tile shapes per job: fixed (opts tile_w x tile_h, default 8x8) or
//     picked per resolution class by the autotuner (rcmvs_autotune);
//   * job order: longest tiles first (pixels per tile x support views), so
//     the blocks of the costliest jobs start first and the short ones fill
//     the tail (longest-processing-time order);
//   * the schedule init -> 2*max(sweeps,1) Jacobi passes -> gate, as plain
//     launches (block b = tile b), as persistent (view, tile) work-queue
//     launches, and/or replayed from a CUDA graph cached on the scene.
// Every variant computes each pixel exactly as the reference does, so all of
// them give the same bits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "ctx_internal.cuh"

namespace rcmvs {

namespace {

int sfail(rcmvs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

#define SCK(x)                                                                                  \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess)                                                                  \
            return sfail(ctx, e_ == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,    \
                         std::string(#x) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

// stereo.rs:275-277: the per-pass perturbation scales, with the host libm's
// powf as in the reference.
float powf_host(float b, float e) { return powf(b, e); }

bool shape_ok(TileShape ts) { return tile_shape_ok(ts); }
// launch_init's kernel for the option flags: 1 one candidate at a time, 0 the
// row-step sweep, 2 the table sweep (the default: 3x faster on C5).
int init_variant(uint32_t flags) {
    if (flags & RCMVS_FLAG_ONE_CANDIDATE) return 1;
    return (flags & RCMVS_FLAG_ROW_STEP_INIT) ? 0 : 2;
}
// Split passes (5 lanes per pixel): at most 128 pixels, so a block of
// split_threads(px) threads at the kernel's 80 registers fits an SM.
bool split_shape_ok(TileShape ts) { return tile_shape_ok(ts) && ts.tw * ts.th <= 128; }
TileShape fixed_shape(const rcmvs_options* o) { return default_tile_shape(o); }

const rcmvs_tune_entry* find_class(const rcmvs_ctx* ctx, int w, int h) {
    for (const auto& e : ctx->tuned)
        if (e.w == w && e.h == h) return &e;
    return nullptr;
}

// Candidate shapes of the autotuner (pixels per tile <= 256, the block size
// the stereo kernels are compiled for); the first one is the default.
// Smaller blocks cost more halo loads per pixel but free their slot sooner.
const TileShape kCandidates[] = {{8, 8},  {16, 4}, {4, 16}, {16, 16}, {32, 8}, {8, 32}, {64, 4},
                                 {16, 8}, {8, 16}, {32, 4}, {8, 4},   {4, 8},  {16, 2}};
constexpr int kNumCandidates = sizeof(kCandidates) / sizeof(kCandidates[0]);

// Fills b for jobs with shapes shp (caller's order), then sorts launch order.
int assemble(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, const std::vector<TileShape>& shp,
             bool lpt, StereoBatch& b) {
    b.order.resize(n_jobs);
    std::iota(b.order.begin(), b.order.end(), 0);
    if (lpt)
        std::stable_sort(b.order.begin(), b.order.end(), [&](int a, int c) {
            const long long ka = (long long)shp[a].tw * shp[a].th * jobs[a].n_src;
            const long long kc = (long long)shp[c].tw * shp[c].th * jobs[c].n_src;
            return ka > kc;
        });
    b.jobs.resize(n_jobs);
    b.start.resize(n_jobs + 1);
    int64_t tiles = 0;
    int nthr = 0;
    size_t smem = 0;
    for (int p = 0; p < n_jobs; ++p) {
        const int j = b.order[p];
        fill_job(sc, jobs[j].ref_idx, jobs[j].srcs, jobs[j].n_src, jobs[j].zmin, jobs[j].zmax, shp[j], b.jobs[p]);
        b.jobs[p].tile_base = (int32_t)tiles;
        b.start[p] = (int32_t)tiles;
        tiles += b.jobs[p].tiles;
        nthr = std::max(nthr, shp[j].tw * shp[j].th);
        smem = std::max(smem, stereo_smem_bytes(shp[j]));
    }
    if (tiles > INT32_MAX) return sfail(ctx, RCMVS_E_LIMIT, "too many tiles in one batch");
    b.start[n_jobs] = (int32_t)tiles;
    b.geom = LaunchGeom{nthr, smem, (int)tiles, nullptr};
    // the streamed passes' own tiling of the same jobs, in launch order
    b.sstart.resize(n_jobs + 1);
    int64_t stiles = 0;
    for (int p = 0; p < n_jobs; ++p) {
        b.sstart[p] = (int32_t)stiles;
        stiles += stream_tiles(b.jobs[p].w, b.jobs[p].h);
    }
    if (stiles > INT32_MAX) return sfail(ctx, RCMVS_E_LIMIT, "too many tiles in one batch");
    b.sstart[n_jobs] = (int32_t)stiles;
    b.sgeom = stream_geom((int)stiles);
    return RCMVS_OK;
}

// Plane-sweep init and one pass over jobs with every job at shape ts, timed
// separately; *ms = the schedule's estimate, init + 2*max(sweeps,1) passes.
int trial(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, const rcmvs_options* opts, TileShape ts,
          int tpp, cudaEvent_t e0, cudaEvent_t e1, cudaEvent_t e2, float* ms) {
    StereoBatch b;
    std::vector<TileShape> shp(n_jobs, ts);
    int rc = assemble(ctx, sc, jobs, n_jobs, shp, false, b);
    if (rc) return rc;
    b.geom.tpp = tpp;
    void *pj, *ps;
    SCK(sc->arena.get(kSlotTuneJobs, sizeof(DevJob) * n_jobs, &pj));
    SCK(sc->arena.get(kSlotTuneStart, sizeof(int32_t) * (n_jobs + 1), &ps));
    cudaStream_t st = ctx->stream;
    SCK(cudaMemcpyAsync(pj, b.jobs.data(), sizeof(DevJob) * n_jobs, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(ps, b.start.data(), sizeof(int32_t) * (n_jobs + 1), cudaMemcpyHostToDevice, st));
    const DevJob* dj = (const DevJob*)pj;
    const int32_t* dst = (const int32_t*)ps;
    const int nh = (int)std::max<uint32_t>(opts->num_hyp, 2u);
    const int variant = init_variant(opts->flags);
    const bool skip_dup = !(opts->flags & RCMVS_FLAG_NO_SKIP_DUPLICATES);
    PlaneBuf A{sc->plane_a, sc->pcost_a, skip_dup ? sc->pd_a : nullptr};
    PlaneBuf B{sc->plane_b, sc->pcost_b, skip_dup ? sc->pd_b : nullptr};
    SCK(cudaEventRecord(e0, st));
    SCK(launch_init(dj, dst, n_jobs, b.geom, nh, sc->census, sc->rays, A, nullptr, st, variant));
    SCK(cudaEventRecord(e1, st));
    const float sig_inv = 0.02f * powf_host(0.28f, 0.0f), sig_n = 0.30f * powf_host(0.42f, 0.0f);
    SCK(launch_pass(dj, dst, n_jobs, b.geom, 0, sig_inv, sig_n, sc->census, sc->rays, A, B, nullptr, st));
    SCK(cudaEventRecord(e2, st));
    SCK(cudaEventSynchronize(e2));
    float t_init = 0.f, t_pass = 0.f;
    SCK(cudaEventElapsedTime(&t_init, e0, e1));
    SCK(cudaEventElapsedTime(&t_pass, e1, e2));
    const uint64_t np = rcmvs_pass_count(opts);
    *ms = t_init + (float)(np ? np : 2) * t_pass;
    return RCMVS_OK;
}

// Tunes the classes of jobs missing from ctx->tuned.
int tune_missing(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, const rcmvs_options* opts) {
    // classes in first-appearance order, each with its first jobs up to ~1 Mpx
    struct Class {
        int w, h;
        std::vector<rcmvs_job> jobs;
        int64_t px = 0;
        float ms[2][kNumCandidates];  // [one thread per pixel, split passes][shape]
    };
    std::vector<Class> cls;
    for (int j = 0; j < n_jobs; ++j) {
        const DevView& V = sc->views[jobs[j].ref_idx];
        if (find_class(ctx, V.w, V.h)) continue;
        Class* c = nullptr;
        for (auto& k : cls)
            if (k.w == V.w && k.h == V.h) c = &k;
        if (!c) {
            cls.push_back(Class{V.w, V.h, {}, 0, {}});
            c = &cls.back();
        }
        if (c->px < (1 << 20)) {
            c->jobs.push_back(jobs[j]);
            c->px += (int64_t)V.w * V.h;
        }
    }
    if (cls.empty()) return RCMVS_OK;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            for (auto& f : ev)
                if (f) cudaEventDestroy(f);
            return sfail(ctx, RCMVS_E_CUDA, "cudaEventCreate failed");
        }
    int rc = RCMVS_OK;
    for (auto& c : cls) {
        float warm = 0.f;  // first launch of a class pays for cold caches
        rc = trial(ctx, sc, c.jobs.data(), (int)c.jobs.size(), opts, kCandidates[0], 1, ev[0], ev[1], ev[2], &warm);
        for (int t = 0; t < 2 && rc == RCMVS_OK; ++t)
            for (int k = 0; k < kNumCandidates && rc == RCMVS_OK; ++k) {
                c.ms[t][k] = INFINITY;
                if (t == 1 && !split_shape_ok(kCandidates[k])) continue;
                for (int rep = 0; rep < 2 && rc == RCMVS_OK; ++rep) {
                    float ms = 0.f;
                    rc = trial(ctx, sc, c.jobs.data(), (int)c.jobs.size(), opts, kCandidates[k], t ? 5 : 1, ev[0],
                               ev[1], ev[2], &ms);
                    c.ms[t][k] = std::min(c.ms[t][k], ms);
                }
            }
        if (rc) break;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    if (ctx->tune_nthr == 0) {  // the (thread count, threads per pixel) with the least summed best time
        double best_sum = INFINITY;
        for (int t = 0; t < 2; ++t)
            for (int nthr : {64, 256, 128, 32}) {
                double sum = 0;
                for (const auto& c : cls) {
                    float m = INFINITY;
                    for (int k = 0; k < kNumCandidates; ++k)
                        if (kCandidates[k].tw * kCandidates[k].th == nthr) m = std::min(m, c.ms[t][k]);
                    sum += m;
                }
                if (sum < best_sum) {
                    best_sum = sum;
                    ctx->tune_nthr = nthr;
                    ctx->tune_tpp = t ? 5 : 1;
                }
            }
    }
    const int t = ctx->tune_tpp == 5 ? 1 : 0;
    for (const auto& c : cls) {
        int kb = -1;
        for (int k = 0; k < kNumCandidates; ++k)
            if (kCandidates[k].tw * kCandidates[k].th == ctx->tune_nthr && (kb < 0 || c.ms[t][k] < c.ms[t][kb])) kb = k;
        if (!(c.ms[t][kb] < INFINITY)) {  // no split shape of this thread count: one thread per pixel
            return sfail(ctx, RCMVS_E_STATE, "autotuner: no tile shape of the chosen kind for a class");
        }
        rcmvs_tune_entry e;
        std::memset(&e, 0, sizeof(e));
        e.w = c.w;
        e.h = c.h;
        e.tile_w = kCandidates[kb].tw;
        e.tile_h = kCandidates[kb].th;
        e.threads_per_pixel = ctx->tune_tpp;
        e.ms_best = c.ms[t][kb];
        e.ms_default = c.ms[0][0];
        ctx->tuned.push_back(e);
    }
    return RCMVS_OK;
}

void append(std::vector<unsigned char>& k, const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    k.insert(k.end(), c, c + n);
}
template <typename T>
void append(std::vector<unsigned char>& k, const T& v) {
    append(k, &v, sizeof(T));
}

}  // namespace

// mvs/src/stereo.rs:131-132 in f64, cast to f32 (RefWorkspace::new)
void rel_pose(const HostCam& r, const HostCam& s, float* rs, float* ts) {
    double rs64[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            rs64[3 * i + j] = s.R[3 * i] * r.R[3 * j] + s.R[3 * i + 1] * r.R[3 * j + 1] + s.R[3 * i + 2] * r.R[3 * j + 2];
    for (int i = 0; i < 9; ++i) rs[i] = (float)rs64[i];
    for (int i = 0; i < 3; ++i) {
        double rt = rs64[3 * i] * r.t[0] + rs64[3 * i + 1] * r.t[1] + rs64[3 * i + 2] * r.t[2];
        ts[i] = (float)(s.t[i] - rt);
    }
}

void fill_job(const rcmvs_scene* sc, int ref, const int32_t* srcs, int n_src, double zmin, double zmax, TileShape ts,
              DevJob& J) {
    std::memset(&J, 0, sizeof(J));
    const DevView& V = sc->views[ref];
    J.view = ref;
    J.nsrc = n_src;
    J.w = V.w;
    J.h = V.h;
    J.off = V.off;
    J.zmin = (float)zmin;
    J.zmax = (float)zmax;
    J.inv_min = 1.0f / J.zmax;  // stereo.rs:248-249 (f32)
    J.inv_max = 1.0f / J.zmin;
    J.tw = ts.tw;
    J.th = ts.th;
    J.tiles_x = (V.w + ts.tw - 1) / ts.tw;
    J.tiles_y = (V.h + ts.th - 1) / ts.th;
    J.tiles = J.tiles_x * J.tiles_y;
    for (int s = 0; s < n_src; ++s) {
        const HostCam& c = sc->cams[srcs[s]];
        DevSrc& D = J.src[s];
        rel_pose(sc->cams[ref], c, D.rs, D.ts);
        D.f = (float)c.f;
        D.cx = (float)c.cx;
        D.cy = (float)c.cy;
        D.k = (float)c.k;
        D.w = sc->views[srcs[s]].w;
        D.h = sc->views[srcs[s]].h;
        D.off = sc->views[srcs[s]].off;
    }
}

int build_batch(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, const rcmvs_options* opts,
                StereoBatch& b) {
    std::vector<TileShape> shp(n_jobs, fixed_shape(opts));
    int tpp = opts->threads_per_pixel <= 1 ? 1 : (int)opts->threads_per_pixel;
    if (tpp != 1 && tpp != 5) return sfail(ctx, RCMVS_E_ARG, "threads_per_pixel must be 0, 1 or 5");
    if (opts->flags & RCMVS_FLAG_AUTOTUNE) {
        int rc = tune_missing(ctx, sc, jobs, n_jobs, opts);
        if (rc) return rc;
        for (int j = 0; j < n_jobs; ++j) {
            const DevView& V = sc->views[jobs[j].ref_idx];
            const rcmvs_tune_entry* e = find_class(ctx, V.w, V.h);
            if (e) shp[j] = TileShape{e->tile_w, e->tile_h};
        }
        tpp = ctx->tune_tpp;
    } else if (!shape_ok(shp[0])) {
        return sfail(ctx, RCMVS_E_ARG, "tile shape must have tw*th <= 256 threads, a multiple of 32");
    } else if (tpp == 5 && !split_shape_ok(shp[0])) {
        return sfail(ctx, RCMVS_E_ARG, "threads_per_pixel 5 takes tiles of at most 128 pixels");
    }
    int rc = assemble(ctx, sc, jobs, n_jobs, shp, true, b);
    b.geom.tpp = tpp;
    b.stream = tpp == 1 && !(opts->flags & RCMVS_FLAG_LOCKSTEP_PASSES);
    return rc;
}

void drop_graph(rcmvs_scene* sc) {
    if (sc->graph) cudaGraphExecDestroy(sc->graph);
    sc->graph = nullptr;
    sc->graph_key.clear();
}

int run_batch(rcmvs_ctx* ctx, rcmvs_scene* sc, const StereoBatch& b, const Schedule& s) {
    const int n_jobs = (int)b.jobs.size();
    if (n_jobs == 0 || b.geom.tiles == 0) return RCMVS_OK;
    cudaStream_t st = ctx->stream;
    void *pj, *ps, *pq = nullptr;
    SCK(sc->arena.get(kSlotJobs, sizeof(DevJob) * n_jobs, &pj));
    SCK(sc->arena.get(kSlotJobStart, sizeof(int32_t) * (n_jobs + 1), &ps));
    const int n_launch = 1 + (int)s.n_passes;
    // the streamed passes are always persistent (each block owns a slice of
    // the scratch), so their launches take queue counters too
    if (s.persistent || b.stream) SCK(sc->arena.get(kSlotQueue, sizeof(unsigned int) * n_launch, &pq));
    // pageable -> device copies return once the host data has been staged
    SCK(cudaMemcpyAsync(pj, b.jobs.data(), sizeof(DevJob) * n_jobs, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(ps, b.start.data(), sizeof(int32_t) * (n_jobs + 1), cudaMemcpyHostToDevice, st));
    void *pss = nullptr, *pscr = nullptr;
    LaunchGeom sgeom = b.sgeom;
    if (b.stream) {
        SCK(sc->arena.get(kSlotStreamStart, sizeof(int32_t) * (n_jobs + 1), &pss));
        SCK(cudaMemcpyAsync(pss, b.sstart.data(), sizeof(int32_t) * (n_jobs + 1), cudaMemcpyHostToDevice, st));
        sgeom.scratch_blocks = std::min(stream_grid(sgeom), sgeom.tiles);
        SCK(sc->arena.get(kSlotStreamScratch, stream_scratch_bytes(sgeom.scratch_blocks), &pscr));
        sgeom.scratch = (float4*)pscr;
    }
    const DevJob* dj = (const DevJob*)pj;
    const int32_t* dst = (const int32_t*)ps;
    // the passes' tile starts and geometry (the streamed tiling by default)
    const int32_t* pst = b.stream ? (const int32_t*)pss : dst;
    unsigned int* queue = (unsigned int*)pq;
    // pass flags (the repeat skip) only with the duplicate skip: both off is
    // the reference's own call sequence
    const bool repeat = s.skip_duplicates && s.repeat_skip;
    PlaneBuf A0{sc->plane_a, sc->pcost_a, s.skip_duplicates ? sc->pd_a : nullptr, repeat ? sc->pf_a : nullptr};
    PlaneBuf B0{sc->plane_b, sc->pcost_b, s.skip_duplicates ? sc->pd_b : nullptr, repeat ? sc->pf_b : nullptr};
    std::vector<float> sig(2 * s.n_passes);
    for (uint64_t pass = 0; pass < s.n_passes; ++pass) {
        const float t = (float)pass / (float)s.n_passes;  // stereo.rs:275-277
        sig[2 * pass] = 0.02f * powf_host(0.28f, t * 4.0f);
        sig[2 * pass + 1] = 0.30f * powf_host(0.42f, t * 4.0f);
    }
    const bool use_graph = s.graph && !ctx->timing;
    const SpanHook hk = use_graph ? SpanHook{} : ctx->hook();

    auto enqueue = [&]() -> cudaError_t {
        cudaError_t e;
        LaunchGeom g = b.geom;
        if (queue && (e = cudaMemsetAsync(queue, 0, sizeof(unsigned int) * n_launch, st))) return e;
        if (s.init == Schedule::LEARNED && s.d_learned &&
            (e = cudaMemsetAsync(s.d_learned, 0, sizeof(unsigned long long), st)))
            return e;
        PlaneBuf A = A0, B = B0;
        g.queue = s.persistent ? queue : nullptr;
        hk.begin(s.init == Schedule::LEARNED ? "learned_init" : "stereo_init");
        if (s.init == Schedule::LEARNED)
            e = launch_init_learned(dj, dst, n_jobs, g, s.nh, sc->census, sc->rays, A, s.pred, s.pred_off,
                                    s.logit_thr, s.n_local, s.span, s.sweep_seeded, s.d_learned, st);
        else
            e = launch_init(dj, dst, n_jobs, g, s.nh, sc->census, sc->rays, A, s.d_work, st,
                            s.init == Schedule::ONE_CANDIDATE ? 1 : (s.init == Schedule::TABLE ? 2 : 0));
        hk.end(s.init == Schedule::LEARNED ? "learned_init" : "stereo_init");
        if (e) return e;
        LaunchGeom gp = b.stream ? sgeom : b.geom;
        for (uint64_t pass = 0; pass < s.n_passes; ++pass) {
            gp.queue = queue ? queue + 1 + pass : nullptr;
            hk.begin("stereo_pass");
            PlaneBuf P = A;
            if (pass == 0) P.flag = nullptr;  // the init leaves no pass flags
            e = launch_pass(dj, pst, n_jobs, gp, pass, sig[2 * pass], sig[2 * pass + 1], sc->census, sc->rays, P, B,
                            s.d_work, st);
            hk.end("stereo_pass");
            if (e) return e;
            std::swap(A, B);
        }
        g.queue = nullptr;
        hk.begin("stereo_gate");
        e = launch_gate(dj, dst, n_jobs, g, s.cost_thr, sc->census, A, sc->depth, sc->cost, sc->normal, st);
        hk.end("stereo_gate");
        return e;
    };

    if (!use_graph) {
        SCK(enqueue());
        return RCMVS_OK;
    }
    // key: everything the captured launches read from the host side
    std::vector<unsigned char> key;
    append(key, b.jobs.data(), sizeof(DevJob) * n_jobs);
    append(key, b.start.data(), sizeof(int32_t) * (n_jobs + 1));
    append(key, b.geom.nthr);
    append(key, b.geom.smem);
    append(key, b.geom.tpp);
    append(key, b.stream);
    append(key, b.sstart.data(), sizeof(int32_t) * (n_jobs + 1));
    append(key, sgeom.scratch_blocks);
    append(key, (int)s.init);
    append(key, s.nh);
    append(key, s.n_passes);
    append(key, s.cost_thr);
    append(key, s.logit_thr);
    append(key, s.n_local);
    append(key, s.span);
    append(key, s.sweep_seeded);
    const void* ptrs[] = {pj, ps, pss, pscr, pq, s.d_work, s.pred, s.pred_off, s.d_learned, sc->census, sc->rays,
                          sc->plane_a, sc->plane_b, sc->pcost_a, sc->pcost_b, A0.d, B0.d, A0.flag, B0.flag,
                          sc->depth, sc->cost, sc->normal};
    append(key, ptrs, sizeof(ptrs));
    if (!sc->graph || key != sc->graph_key) {
        drop_graph(sc);
        SCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const cudaError_t le = enqueue();
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(st, &graph);
        if (le != cudaSuccess || ce != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            SCK(le != cudaSuccess ? le : ce);
        }
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        SCK(ie);
        sc->graph = exec;
        sc->graph_key.swap(key);
    }
    SCK(cudaGraphLaunch(sc->graph, st));
    return RCMVS_OK;
}

bool tile_shape_ok(TileShape ts) {
    return ts.tw > 0 && ts.th > 0 && ts.tw * ts.th <= 256 && (ts.tw * ts.th) % 32 == 0 &&
           stereo_smem_bytes(ts) <= 48 * 1024;
}

// Default tile: 8x8 measured fastest among the fixed shapes at 960x720 (K 8),
// 1920x1080 (K 10) and mixed batches (K 4-12) on B200, 4-7% ahead of 16x16:
// a block holds its SM slot until its slowest warp (the one with the fewest
// early aborts) is done, and smaller blocks release it sooner.
TileShape default_tile_shape(const rcmvs_options* o) {
    if (o && o->tile_w > 0 && o->tile_h > 0) return TileShape{(int)o->tile_w, (int)o->tile_h};
    return TileShape{8, 8};
}

}  // namespace rcmvs

using namespace rcmvs;

extern "C" {

int rcmvs_autotune(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int32_t n_jobs,
                   const rcmvs_options* opts) {
    if (!ctx || !sc || !opts || n_jobs < 0 || (n_jobs > 0 && !jobs))
        return sfail(ctx, RCMVS_E_ARG, "rcmvs_autotune: bad argument");
    if (sc->ctx != ctx) return sfail(ctx, RCMVS_E_ARG, "scene belongs to another context");
    for (int j = 0; j < n_jobs; ++j) {
        if (jobs[j].ref_idx < 0 || jobs[j].ref_idx >= sc->n_views || jobs[j].n_src < 0 ||
            jobs[j].n_src > RCMVS_MAX_SOURCES || (jobs[j].n_src > 0 && !jobs[j].srcs))
            return sfail(ctx, RCMVS_E_ARG, "rcmvs_autotune: bad job");
        for (int q = 0; q < jobs[j].n_src; ++q)
            if (jobs[j].srcs[q] < 0 || jobs[j].srcs[q] >= sc->n_views)
                return sfail(ctx, RCMVS_E_ARG, "rcmvs_autotune: bad source");
        if (!(jobs[j].zmin > 0 && jobs[j].zmax > 0 && std::isfinite(jobs[j].zmin) && std::isfinite(jobs[j].zmax)))
            return sfail(ctx, RCMVS_E_ARG, "rcmvs_autotune: bad depth range");
    }
    SCK(cudaSetDevice(ctx->device));
    return tune_missing(ctx, sc, jobs, n_jobs, opts);
}

int rcmvs_tune_table(rcmvs_ctx* ctx, rcmvs_tune_entry* out, int32_t cap, int32_t* n_out) {
    if (!ctx || !n_out || cap < 0 || (cap > 0 && !out)) return sfail(ctx, RCMVS_E_ARG, "rcmvs_tune_table: bad argument");
    const int n = std::min<int>(cap, (int)ctx->tuned.size());
    for (int i = 0; i < n; ++i) out[i] = ctx->tuned[i];
    *n_out = n;
    return RCMVS_OK;
}

int rcmvs_tune_set(rcmvs_ctx* ctx, const rcmvs_tune_entry* entries, int32_t n) {
    if (!ctx || n < 0 || (n > 0 && !entries)) return sfail(ctx, RCMVS_E_ARG, "rcmvs_tune_set: bad argument");
    const int tpp = n > 0 && entries[0].threads_per_pixel == 5 ? 5 : 1;
    for (int i = 0; i < n; ++i) {
        const TileShape ts{entries[i].tile_w, entries[i].tile_h};
        const int t = entries[i].threads_per_pixel <= 1 ? 1 : entries[i].threads_per_pixel;
        if (entries[i].w <= 0 || entries[i].h <= 0 || !shape_ok(ts) || t != tpp || (tpp == 5 && !split_shape_ok(ts)))
            return sfail(ctx, RCMVS_E_ARG, "rcmvs_tune_set: bad entry " + std::to_string(i));
    }
    ctx->tuned.assign(entries, entries + n);
    for (auto& e : ctx->tuned) e.threads_per_pixel = tpp;
    ctx->tune_nthr = n > 0 ? entries[0].tile_w * entries[0].tile_h : 0;
    ctx->tune_tpp = tpp;
    return RCMVS_OK;
}

}  // extern "C"
