// learned_api.cu — C ABI of the learned plane proposals (no reference
// counterpart): the proposal network (parameters, training step, forward),
// the quarter-resolution cost volume of a scene, and stereo seeded by the
// network's predictions.
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "ctx_internal.cuh"
#include "learned.cuh"


using namespace rcmvs;

namespace {

int lfail(rcmvs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

#define LCK(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return lfail(ctx, e_ == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,   \
                         std::string(#x) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

struct Layer {
    int64_t w_off, b_off;  // offsets into the parameter vector
    int cin, cout;
};

std::vector<Layer> layers() {
    std::vector<Layer> L;
    int64_t off = 0;
    for (int l = 0; l < NET_LAYERS; ++l) {
        Layer y;
        y.cin = NET_CIN[l];
        y.cout = NET_COUT[l];
        y.w_off = off;
        off += 9LL * y.cout * y.cin;
        y.b_off = off;
        off += y.cout;
        L.push_back(y);
    }
    return L;
}

int64_t param_count() {
    auto L = layers();
    return L.back().b_off + L.back().cout;
}

// arena slots of the net (activations and scratch)
enum { N_ACT0 = 0, N_OUT = 10, N_DOUT = 11, N_DY0 = 12, N_DY1 = 13, N_FLIP = 14, N_ACC = 15 };

}  // namespace

struct rcmvs_net {
    rcmvs_ctx* ctx = nullptr;
    int64_t n = 0;
    float* p = nullptr;   // f32 master parameters
    float* g = nullptr;   // gradients
    float* m = nullptr;   // Adam moments
    float* v = nullptr;
    uint8_t* mask = nullptr;  // 0 for padded weights / biases
    void* pb = nullptr;   // BF16 copy used by the kernels (biases too, unused)
    float* bias = nullptr;  // f32 biases are read straight from p
    int64_t step = 0;
    DeviceArena arena;
};

extern "C" {

uint64_t rcmvs_net_param_count(void) { return (uint64_t)param_count(); }

int rcmvs_net_create(rcmvs_ctx* ctx, const float* params, uint64_t seed, rcmvs_net** out) {
    if (!ctx || !out) return lfail(ctx, RCMVS_E_ARG, "rcmvs_net_create: bad argument");
    *out = nullptr;
    const int64_t n = param_count();
    std::vector<float> h(n, 0.f);
    std::vector<uint8_t> mk(n, 0);
    auto L = layers();
    std::mt19937_64 rng(seed);
    for (int l = 0; l < NET_LAYERS; ++l) {
        const Layer& y = L[l];
        const float sd = std::sqrt(2.0f / (9.0f * NET_CIN_REAL[l]));  // He initialisation
        std::normal_distribution<float> nd(0.f, sd);
        for (int t = 0; t < 9; ++t)
            for (int co = 0; co < y.cout; ++co)
                for (int ci = 0; ci < y.cin; ++ci) {
                    const int64_t i = y.w_off + ((int64_t)t * y.cout + co) * y.cin + ci;
                    const bool real = co < NET_COUT_REAL[l] && ci < NET_CIN_REAL[l];
                    mk[i] = real;
                    h[i] = real ? nd(rng) : 0.f;
                }
        for (int co = 0; co < y.cout; ++co) {
            mk[y.b_off + co] = co < NET_COUT_REAL[l];
            h[y.b_off + co] = 0.f;
        }
    }
    if (params)
        for (int64_t i = 0; i < n; ++i) h[i] = mk[i] ? params[i] : 0.f;
    rcmvs_net* net = new rcmvs_net();
    net->ctx = ctx;
    net->n = n;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (!e) e = cudaMalloc(&net->p, 4 * n);
    if (!e) e = cudaMalloc(&net->g, 4 * n);
    if (!e) e = cudaMalloc(&net->m, 4 * n);
    if (!e) e = cudaMalloc(&net->v, 4 * n);
    if (!e) e = cudaMalloc(&net->mask, n);
    if (!e) e = cudaMalloc(&net->pb, 2 * n);
    if (!e) e = cudaMemcpy(net->p, h.data(), 4 * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(net->mask, mk.data(), n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemset(net->m, 0, 4 * n);
    if (!e) e = cudaMemset(net->v, 0, 4 * n);
    if (!e) e = launch_to_bf16(net->p, n, net->pb, ctx->stream);
    if (!e) e = cudaStreamSynchronize(ctx->stream);
    if (e) {
        cudaFree(net->p);
        cudaFree(net->g);
        cudaFree(net->m);
        cudaFree(net->v);
        cudaFree(net->mask);
        cudaFree(net->pb);
        delete net;
        return lfail(ctx, RCMVS_E_CUDA, std::string("rcmvs_net_create: ") + cudaGetErrorString(e));
    }
    *out = net;
    return RCMVS_OK;
}

void rcmvs_net_destroy(rcmvs_net* net) {
    if (!net) return;
    cudaSetDevice(net->ctx->device);
    cudaStreamSynchronize(net->ctx->stream);
    cudaFree(net->p);
    cudaFree(net->g);
    cudaFree(net->m);
    cudaFree(net->v);
    cudaFree(net->mask);
    cudaFree(net->pb);
    net->arena.release();
    delete net;
}

int rcmvs_net_get_params(rcmvs_net* net, float* out) {
    if (!net || !out) return RCMVS_E_ARG;
    rcmvs_ctx* ctx = net->ctx;
    LCK(cudaSetDevice(ctx->device));
    LCK(cudaMemcpyAsync(out, net->p, 4 * net->n, cudaMemcpyDeviceToHost, ctx->stream));
    LCK(cudaStreamSynchronize(ctx->stream));
    return RCMVS_OK;
}

}  // extern "C"

namespace {

const void* wb(rcmvs_net* net, const Layer& y) { return (const char*)net->pb + 2 * y.w_off; }

// Forward through all layers; activations Y1..Y5 kept in arena slots
// N_ACT0+1..5 for the backward pass; head output (f32) -> out.
int net_forward(rcmvs_ctx* ctx, rcmvs_net* net, const void* x, int N, int H, int W, float* out) {
    auto L = layers();
    const int64_t npx = (int64_t)N * H * W;
    const void* in = x;
    for (int l = 0; l < NET_LAYERS; ++l) {
        const Layer& y = L[l];
        const float* b = net->p + y.b_off;
        if (l == NET_LAYERS - 1) {
            LCK(launch_conv3x3(y.cin, y.cout, false, true, in, nullptr, N, H, W, wb(net, y), b, out, ctx->stream));
        } else {
            void* act;
            LCK(net->arena.get(N_ACT0 + 1 + l, 2 * npx * y.cout, &act));
            LCK(launch_conv3x3(y.cin, y.cout, true, false, in, nullptr, N, H, W, wb(net, y), b, act, ctx->stream));
            in = act;
        }
    }
    return RCMVS_OK;
}

}  // namespace

extern "C" {

int rcmvs_net_forward(rcmvs_ctx* ctx, rcmvs_net* net, const void* x_dev, int32_t n, int32_t h, int32_t w,
                      float* out_dev) {
    if (!ctx || !net || !x_dev || !out_dev || n <= 0 || h <= 0 || w <= 0)
        return lfail(ctx, RCMVS_E_ARG, "rcmvs_net_forward: bad argument");
    LCK(cudaSetDevice(ctx->device));
    return net_forward(ctx, net, x_dev, n, h, w, out_dev);
}

// One training step: forward, loss, backward; apply != 0 also takes an Adam
// step with learning rate lr.  loss_out (nullable) gets the mean loss over
// valid pixels; grads_host (nullable) the gradient of that mean loss.
int rcmvs_net_train_step(rcmvs_ctx* ctx, rcmvs_net* net, const void* x_dev, const float* labels_dev, int32_t n,
                         int32_t h, int32_t w, float lr, int32_t apply, float* loss_out, float* grads_host) {
    if (!ctx || !net || !x_dev || !labels_dev || n <= 0 || h <= 0 || w <= 0)
        return lfail(ctx, RCMVS_E_ARG, "rcmvs_net_train_step: bad argument");
    LCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    auto L = layers();
    const int64_t npx = (int64_t)n * h * w;
    void *out, *dout, *acc;
    LCK(net->arena.get(N_OUT, 4 * npx * NET_OUT_C, &out));
    LCK(net->arena.get(N_DOUT, 2 * npx * NET_OUT_C, &dout));
    LCK(net->arena.get(N_ACC, 16, &acc));
    int rc = net_forward(ctx, net, x_dev, n, h, w, (float*)out);
    if (rc) return rc;
    LCK(cudaMemsetAsync(acc, 0, 16, st));
    LCK(launch_loss((const float*)out, labels_dev, npx, 1.0f, dout, (float*)acc, st));
    LCK(cudaMemsetAsync(net->g, 0, 4 * net->n, st));
    // backward, last layer first.  dY of layer l is in `dcur` (its pre-ReLU
    // gradient is dY * (Y > 0), applied on load through the mask).
    const void* dcur = dout;
    int flipbuf = 0;
    for (int l = NET_LAYERS - 1; l >= 0; --l) {
        const Layer& y = L[l];
        void* xin = nullptr;
        if (l == 0) {
            xin = const_cast<void*>(x_dev);
        } else {
            LCK(net->arena.get(N_ACT0 + l, 2 * npx * NET_COUT[l - 1], &xin));
        }
        void* ymask = nullptr;  // this layer's ReLU output (none for the head)
        if (l < NET_LAYERS - 1) LCK(net->arena.get(N_ACT0 + 1 + l, 2 * npx * y.cout, &ymask));
        LCK(launch_conv3x3_wgrad(y.cin, y.cout, xin, dcur, ymask, n, h, w, net->g + y.w_off, st));
        LCK(launch_bias_grad(y.cout, dcur, ymask, npx, net->g + y.b_off, st));
        if (l > 0) {
            void *flip, *dnext;
            LCK(net->arena.get(N_FLIP, 2 * 9 * y.cout * y.cin, &flip));
            LCK(launch_flip_weights(wb(net, y), y.cout, y.cin, flip, st));
            LCK(net->arena.get(N_DY0 + flipbuf, 2 * npx * y.cin, &dnext));
            LCK(launch_conv3x3(y.cout, y.cin, false, false, dcur, ymask, n, h, w, flip, nullptr, dnext, st));
            dcur = dnext;
            flipbuf ^= 1;
        }
    }
    float hacc[2];
    LCK(cudaMemcpyAsync(hacc, acc, 8, cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
    const float cnt = hacc[1] > 0.f ? hacc[1] : 1.f;
    if (loss_out) *loss_out = hacc[0] / cnt;
    if (grads_host) {
        LCK(cudaMemcpyAsync(grads_host, net->g, 4 * net->n, cudaMemcpyDeviceToHost, st));
        LCK(cudaStreamSynchronize(st));
        for (int64_t i = 0; i < net->n; ++i) grads_host[i] /= cnt;
    }
    if (apply) {
        net->step++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float bc1 = 1.f - std::pow(b1, (float)net->step), bc2 = 1.f - std::pow(b2, (float)net->step);
        LCK(launch_adam(net->p, net->g, net->m, net->v, net->mask, net->n, lr, b1, b2, 1e-8f, bc1, bc2, 1.f / cnt,
                        net->pb, st));
    }
    return RCMVS_OK;
}

}  // extern "C"

// ------------------------------------------------------------ scene side
namespace {

// quarter-resolution grey, census and rays of every view (once per scene)
int ensure_quarter(rcmvs_ctx* ctx, rcmvs_scene* sc) {
    if (sc->have_quarter) return RCMVS_OK;
    std::vector<DevView> q;
    std::vector<int32_t> blk, tiles;
    std::vector<double> cams;
    int64_t off = 0;
    int nb = 0, nt = 0;
    for (int v = 0; v < sc->n_views; ++v) {
        const int w = sc->views[v].w / 4, h = sc->views[v].h / 4;
        q.push_back(DevView{w, h, off});
        blk.push_back(nb);
        tiles.push_back(nt);
        nb += (int)(((int64_t)w * h + 255) / 256);
        nt += census_tiles(w, h);
        off += (int64_t)w * h;
        // pixel centre of quarter cell X is full-res 4X + 1.5
        const HostCam& c = sc->cams[v];
        cams.insert(cams.end(), {c.f / 4.0, (c.cx - 1.5) / 4.0, (c.cy - 1.5) / 4.0, c.k});
    }
    blk.push_back(nb);
    tiles.push_back(nt);
    sc->qviews = q;
    sc->nq_px = off;
    sc->qblocks = nb;
    sc->qcensus_tiles = nt;
    const size_t np = (size_t)std::max<int64_t>(off, 1);
    cudaStream_t st = ctx->stream;
    rcmvs_ctx::SpareScene& sp = ctx->spare;
    const int nq = (int)q.size();
    // in the order of SpareScene::quarter
    void** qp[7] = {(void**)&sc->gray_q,      (void**)&sc->census_q, (void**)&sc->rays_q,
                    (void**)&sc->d_qviews,    (void**)&sc->d_qtile_start, (void**)&sc->d_qcams,
                    (void**)&sc->d_qblk_start};
    for (void** p : qp) {  // what a failed earlier attempt left
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (sp.quarter[0] && sp.q_cap_px >= np && sp.q_cap_views >= nq) {
        // the last destroyed scene's quarter buffers (every one is written
        // below or by the quarter census before it is read)
        for (int i = 0; i < 7; ++i) {
            *qp[i] = sp.quarter[i];
            sp.quarter[i] = nullptr;
        }
        sc->q_cap_px = sp.q_cap_px;
        sc->q_cap_views = sp.q_cap_views;
        sp.q_cap_px = 0;
        sp.q_cap_views = 0;
    } else {
        LCK(cudaMalloc(&sc->gray_q, np));
        LCK(cudaMalloc(&sc->census_q, 8 * np));
        LCK(cudaMalloc(&sc->rays_q, 8 * np));
        LCK(cudaMalloc(&sc->d_qviews, sizeof(DevView) * q.size()));
        LCK(cudaMalloc(&sc->d_qtile_start, sizeof(int32_t) * tiles.size()));
        LCK(cudaMalloc(&sc->d_qblk_start, sizeof(int32_t) * blk.size()));
        LCK(cudaMalloc(&sc->d_qcams, sizeof(double) * cams.size()));
        sc->q_cap_px = np;
        sc->q_cap_views = nq;
    }
    LCK(cudaMemcpyAsync(sc->d_qviews, q.data(), sizeof(DevView) * q.size(), cudaMemcpyHostToDevice, st));
    LCK(cudaMemcpyAsync(sc->d_qtile_start, tiles.data(), sizeof(int32_t) * tiles.size(), cudaMemcpyHostToDevice, st));
    LCK(cudaMemcpyAsync(sc->d_qblk_start, blk.data(), sizeof(int32_t) * blk.size(), cudaMemcpyHostToDevice, st));
    LCK(cudaMemcpyAsync(sc->d_qcams, cams.data(), sizeof(double) * cams.size(), cudaMemcpyHostToDevice, st));
    LCK(cudaStreamSynchronize(st));
    sc->have_quarter = true;
    return RCMVS_OK;
}

int quarter_prepare(rcmvs_ctx* ctx, rcmvs_scene* sc) {
    int rc = ensure_quarter(ctx, sc);
    if (rc) return rc;
    LCK(launch_downsample4(sc->d_views, sc->d_qviews, sc->d_qblk_start, sc->n_views, sc->qblocks, sc->gray,
                           sc->gray_q, ctx->stream));
    LCK(launch_census_rays(sc->d_qviews, sc->d_qtile_start, sc->n_views, sc->qcensus_tiles, sc->gray_q,
                           sc->census_q, sc->rays_q, sc->d_qcams, ctx->stream));
    return RCMVS_OK;
}

// quarter-resolution jobs (for the cost volume): views, sizes and
// intrinsics of the quarter copies; also returns each job's output offset.
int quarter_jobs(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, DevJob** d_jobs,
                 int32_t** d_blk, int64_t** d_off, int* total_blocks, int64_t* total_px) {
    std::vector<DevJob> hj(n_jobs);
    std::vector<int32_t> blk(n_jobs + 1);
    std::vector<int64_t> off(n_jobs + 1);
    int nb = 0;
    int64_t px = 0;
    for (int j = 0; j < n_jobs; ++j) {
        DevJob& J = hj[j];
        std::memset(&J, 0, sizeof(J));
        const int r = jobs[j].ref_idx;
        const DevView& Q = sc->qviews[r];
        J.view = r;
        J.nsrc = jobs[j].n_src;
        J.w = Q.w;
        J.h = Q.h;
        J.off = Q.off;
        J.zmin = (float)jobs[j].zmin;
        J.zmax = (float)jobs[j].zmax;
        J.inv_min = 1.0f / J.zmax;
        J.inv_max = 1.0f / J.zmin;
        const HostCam& rc = sc->cams[r];
        for (int s = 0; s < J.nsrc; ++s) {
            const int sv = jobs[j].srcs[s];
            const HostCam& c = sc->cams[sv];
            DevSrc& D = J.src[s];
            rel_pose(rc, c, D.rs, D.ts);
            D.f = (float)(c.f / 4.0);
            D.cx = (float)((c.cx - 1.5) / 4.0);
            D.cy = (float)((c.cy - 1.5) / 4.0);
            D.k = (float)c.k;
            D.w = sc->qviews[sv].w;
            D.h = sc->qviews[sv].h;
            D.off = sc->qviews[sv].off;
        }
        blk[j] = nb;
        off[j] = px;
        nb += costvol_tiles(Q.w, Q.h);
        px += (int64_t)Q.w * Q.h;
    }
    blk[n_jobs] = nb;
    off[n_jobs] = px;
    void *pj, *pb, *po;
    LCK(sc->arena.get(40, sizeof(DevJob) * n_jobs, &pj));
    LCK(sc->arena.get(41, sizeof(int32_t) * (n_jobs + 1), &pb));
    LCK(sc->arena.get(42, sizeof(int64_t) * (n_jobs + 1), &po));
    cudaStream_t st = ctx->stream;
    LCK(cudaMemcpyAsync(pj, hj.data(), sizeof(DevJob) * n_jobs, cudaMemcpyHostToDevice, st));
    LCK(cudaMemcpyAsync(pb, blk.data(), sizeof(int32_t) * (n_jobs + 1), cudaMemcpyHostToDevice, st));
    LCK(cudaMemcpyAsync(po, off.data(), sizeof(int64_t) * (n_jobs + 1), cudaMemcpyHostToDevice, st));
    LCK(cudaStreamSynchronize(st));  // host vectors go out of scope
    *d_jobs = (DevJob*)pj;
    *d_blk = (int32_t*)pb;
    *d_off = (int64_t*)po;
    *total_blocks = nb;
    *total_px = px;
    return RCMVS_OK;
}

int check_jobs(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs) {
    if (!jobs || n_jobs <= 0) return lfail(ctx, RCMVS_E_ARG, "empty job list");
    for (int j = 0; j < n_jobs; ++j) {
        if (jobs[j].ref_idx < 0 || jobs[j].ref_idx >= sc->n_views || jobs[j].n_src < 0 ||
            jobs[j].n_src > RCMVS_MAX_SOURCES || (jobs[j].n_src > 0 && !jobs[j].srcs))
            return lfail(ctx, RCMVS_E_ARG, "bad job");
        for (int s = 0; s < jobs[j].n_src; ++s)
            if (jobs[j].srcs[s] < 0 || jobs[j].srcs[s] >= sc->n_views) return lfail(ctx, RCMVS_E_ARG, "bad source");
        if (!(jobs[j].zmin > 0 && jobs[j].zmax > 0 && std::isfinite(jobs[j].zmin) && std::isfinite(jobs[j].zmax)))
            return lfail(ctx, RCMVS_E_ARG, "bad depth range");
    }
    return RCMVS_OK;
}

constexpr uint32_t kSeedFlags = RCMVS_FLAG_PERSISTENT | RCMVS_FLAG_CUDA_GRAPH | RCMVS_FLAG_AUTOTUNE |
                               RCMVS_FLAG_NO_SKIP_DUPLICATES | RCMVS_FLAG_INIT_ONLY | RCMVS_FLAG_SEED_AND_SWEEP |
                               RCMVS_FLAG_NO_REPEAT_SKIP | RCMVS_FLAG_LOCKSTEP_PASSES |
                               RCMVS_FLAG_ROW_STEP_INIT;  // the learned init has its own sweep: no effect here

int check_seed_args(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, const rcmvs_options* opts,
                    float conf_thr, int n_local, float span) {
    if (n_local < 1 || n_local > 256 || !(span >= 0.f && span <= 1.f) || std::isnan(conf_thr))
        return lfail(ctx, RCMVS_E_ARG, "learned init: n_local must be 1..256, span in [0, 1], conf_thr a number");
    if (opts->flags & ~kSeedFlags) return lfail(ctx, RCMVS_E_ARG, "learned init: unsupported bits in opts->flags");
    if (opts->passes > RCMVS_MAX_PASSES) return lfail(ctx, RCMVS_E_ARG, "opts->passes above RCMVS_MAX_PASSES");
    if (sc->ctx != ctx) return lfail(ctx, RCMVS_E_ARG, "scene belongs to another context");
    return check_jobs(ctx, sc, jobs, n_jobs);
}

// The confidence test sigmoid(logit) >= conf_thr as a threshold on the
// logit: ln(c / (1 - c)) in f64, rounded to f32; -inf for c <= 0 (every
// finite logit passes), +inf for c >= 1 (none does).
float logit_threshold(float conf_thr) {
    if (!(conf_thr > 0.0f)) return -INFINITY;
    if (!(conf_thr < 1.0f)) return INFINITY;
    const double c = (double)conf_thr;
    return (float)std::log(c / (1.0 - c));
}

struct QuarterDims {
    int w, h;
};
QuarterDims quarter_dims(const rcmvs_scene* sc, int view) {
    return QuarterDims{sc->views[view].w >> 2, sc->views[view].h >> 2};
}

// The full-resolution stereo batch with the learned init from `pred` (the
// jobs' quarter-resolution predictions back to back, device memory).
int seeded_stereo(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int n_jobs, const rcmvs_options* opts,
                  const float* pred, float conf_thr, int n_local, float span, uint64_t* learned_pixels) {
    cudaStream_t st = ctx->stream;
    StereoBatch batch;
    int rc = build_batch(ctx, sc, jobs, n_jobs, opts, batch);
    if (rc) return rc;
    std::vector<int64_t> qoff(n_jobs), poff(n_jobs);
    for (int j = 0, o = 0; j < n_jobs; ++j) {
        qoff[j] = o;
        const QuarterDims q = quarter_dims(sc, jobs[j].ref_idx);
        o += (int64_t)q.w * q.h;
    }
    for (int p = 0; p < n_jobs; ++p) poff[p] = qoff[batch.order[p]];
    void *ppo, *pcnt;
    LCK(sc->arena.get(46, sizeof(int64_t) * n_jobs, &ppo));
    LCK(sc->arena.get(47, 16, &pcnt));
    LCK(cudaMemcpyAsync(ppo, poff.data(), sizeof(int64_t) * n_jobs, cudaMemcpyHostToDevice, st));
    Schedule sched;
    sched.init = Schedule::LEARNED;
    sched.nh = (int)std::max<uint32_t>(opts->num_hyp, 2u);
    sched.n_passes = rcmvs_pass_count(opts);
    sched.cost_thr = opts->cost_thr;
    sched.persistent = (opts->flags & RCMVS_FLAG_PERSISTENT) != 0;
    sched.graph = (opts->flags & RCMVS_FLAG_CUDA_GRAPH) != 0;
    sched.skip_duplicates = !(opts->flags & RCMVS_FLAG_NO_SKIP_DUPLICATES);
    sched.repeat_skip = !(opts->flags & RCMVS_FLAG_NO_REPEAT_SKIP);
    sched.pred = pred;
    sched.pred_off = (const int64_t*)ppo;
    sched.logit_thr = logit_threshold(conf_thr);
    sched.n_local = n_local;
    sched.span = span;
    sched.sweep_seeded = (opts->flags & RCMVS_FLAG_SEED_AND_SWEEP) != 0;
    sched.d_learned = (unsigned long long*)pcnt;
    rc = run_batch(ctx, sc, batch, sched);
    if (rc) return rc;
    for (int j = 0; j < n_jobs; ++j) sc->has_depth[jobs[j].ref_idx] = 1;
    if (learned_pixels) {
        unsigned long long h = 0;
        LCK(cudaMemcpyAsync(&h, pcnt, 8, cudaMemcpyDeviceToHost, st));
        LCK(cudaStreamSynchronize(st));
        *learned_pixels = h;
    }
    return RCMVS_OK;
}

}  // namespace

extern "C" {

int rcmvs_scene_costvol(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int32_t n_jobs, void* out_dev) {
    if (!ctx || !sc || !out_dev) return lfail(ctx, RCMVS_E_ARG, "rcmvs_scene_costvol: bad argument");
    int rc = check_jobs(ctx, sc, jobs, n_jobs);
    if (rc) return rc;
    LCK(cudaSetDevice(ctx->device));
    rc = quarter_prepare(ctx, sc);
    if (rc) return rc;
    DevJob* dj;
    int32_t* db;
    int64_t* doff;
    int nb;
    int64_t px;
    rc = quarter_jobs(ctx, sc, jobs, n_jobs, &dj, &db, &doff, &nb, &px);
    if (rc) return rc;
    LCK(launch_costvol(dj, db, n_jobs, nb, doff, sc->census_q, sc->rays_q, sc->gray_q, out_dev, ctx->stream));
    return RCMVS_OK;
}

// Stereo seeded by the network: cost volume -> network -> learned init (sweep
// fallback below conf_thr) -> 2*max(sweeps,1) Jacobi passes -> gate.
int rcmvs_scene_estimate_depth_learned(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int32_t n_jobs,
                                       const rcmvs_options* opts, rcmvs_net* net, float conf_thr,
                                       int32_t n_local, float span, uint64_t* learned_pixels) {
    if (!ctx || !sc || !opts || !net)
        return lfail(ctx, RCMVS_E_ARG, "rcmvs_scene_estimate_depth_learned: bad argument");
    int rc = check_seed_args(ctx, sc, jobs, n_jobs, opts, conf_thr, n_local, span);
    if (rc) return rc;
    LCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const SpanHook hk = ctx->hook();
    hk.begin("learned_costvol");
    rc = quarter_prepare(ctx, sc);
    if (rc) return rc;
    DevJob* dqj;
    int32_t* dqb;
    int64_t* dqoff;
    int qnb;
    int64_t qpx;
    rc = quarter_jobs(ctx, sc, jobs, n_jobs, &dqj, &dqb, &dqoff, &qnb, &qpx);
    if (rc) return rc;
    void *cv, *pred;
    LCK(sc->arena.get(43, 2 * (size_t)qpx * COSTVOL_C, &cv));
    LCK(sc->arena.get(44, 4 * (size_t)qpx * NET_OUT_C, &pred));
    LCK(launch_costvol(dqj, dqb, n_jobs, qnb, dqoff, sc->census_q, sc->rays_q, sc->gray_q, cv, st));
    hk.end("learned_costvol");
    // network, one launch sequence per group of jobs with equal quarter size
    hk.begin("learned_net");
    {
        std::vector<int64_t> off(n_jobs);
        int64_t o = 0;
        for (int j = 0; j < n_jobs; ++j) {
            off[j] = o;
            o += (int64_t)sc->qviews[jobs[j].ref_idx].w * sc->qviews[jobs[j].ref_idx].h;
        }
        int j = 0;
        while (j < n_jobs) {
            const DevView& Q = sc->qviews[jobs[j].ref_idx];
            int e = j + 1;
            while (e < n_jobs && sc->qviews[jobs[e].ref_idx].w == Q.w && sc->qviews[jobs[e].ref_idx].h == Q.h) ++e;
            if (Q.w > 0 && Q.h > 0)
                rc = net_forward(ctx, net, (const char*)cv + 2 * off[j] * COSTVOL_C, e - j, Q.h, Q.w,
                                 (float*)pred + off[j] * NET_OUT_C);
            if (rc) return rc;
            j = e;
        }
    }
    hk.end("learned_net");
    return seeded_stereo(ctx, sc, jobs, n_jobs, opts, (const float*)pred, conf_thr, n_local, span, learned_pixels);
}

// Stereo seeded by caller-given proposals (the network's output format).
int rcmvs_scene_estimate_depth_seeded(rcmvs_ctx* ctx, rcmvs_scene* sc, const rcmvs_job* jobs, int32_t n_jobs,
                                      const rcmvs_options* opts, const float* pred, int32_t pred_on_device,
                                      float conf_thr, int32_t n_local, float span, uint64_t* learned_pixels) {
    if (!ctx || !sc || !opts || !pred)
        return lfail(ctx, RCMVS_E_ARG, "rcmvs_scene_estimate_depth_seeded: bad argument");
    int rc = check_seed_args(ctx, sc, jobs, n_jobs, opts, conf_thr, n_local, span);
    if (rc) return rc;
    LCK(cudaSetDevice(ctx->device));
    if (!pred_on_device) {
        int64_t qpx = 0;
        for (int j = 0; j < n_jobs; ++j) {
            const QuarterDims q = quarter_dims(sc, jobs[j].ref_idx);
            qpx += (int64_t)q.w * q.h;
        }
        void* dp;
        LCK(sc->arena.get(44, 4 * (size_t)std::max<int64_t>(qpx, 1) * NET_OUT_C, &dp));
        LCK(cudaMemcpyAsync(dp, pred, 4 * (size_t)qpx * NET_OUT_C, cudaMemcpyHostToDevice, ctx->stream));
        pred = (const float*)dp;
    }
    return seeded_stereo(ctx, sc, jobs, n_jobs, opts, pred, conf_thr, n_local, span, learned_pixels);
}

}  // extern "C"
