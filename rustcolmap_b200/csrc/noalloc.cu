// noalloc.cu — estimate_depth for callers that cannot allocate device memory.
//
// Some callers of this library are not allowed to call cudaMalloc: a host
// application whose GPU memory is owned by another allocator (a framework's
// caching pool, an engine with a fixed budget), or a real-time loop that must
// not take the device-wide synchronisation that cudaMalloc/cudaFree imply.
// rcmvs_estimate_depth_noalloc serves them.  It takes device pointers for
// its inputs and outputs and keeps every intermediate buffer (grey copies,
// census, rays, double-buffered planes, job descriptors) in one file-scope
// __device__ array of fixed size, RCMVS_NOALLOC_SCRATCH_BYTES.
//
// The array lives in this translation unit's own module.  Under CUDA's
// default lazy module loading a device reserves it the first time this entry
// point runs there (eager loading reserves it on every device that loads the
// library) and holds it until the process exits.  Every call on a device
// shares the array and leaves its contents behind; the kernels write every
// element they later read, so nothing has to be cleared between calls.
// Calls whose GPU work overlaps (two streams, or two host threads) race on
// the array: serialise them.
#include <cstring>

#include "rcmvs_internal.cuh"


using namespace rcmvs;

namespace {

constexpr int kViews = 1 + RCMVS_NOALLOC_MAX_SOURCES;
constexpr size_t kPx = RCMVS_NOALLOC_MAX_PIXELS;
constexpr size_t kDesc = 16384;  // DevView[], tile starts, cameras, DevJob, job start
constexpr size_t al(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kOffGray = kDesc;
constexpr size_t kOffCensus = kOffGray + al(kViews * kPx);
constexpr size_t kOffRays = kOffCensus + al(kViews * kPx * 8);
constexpr size_t kOffPlaneA = kOffRays + al(kViews * kPx * 8);
constexpr size_t kOffPlaneB = kOffPlaneA + al(kPx * 16);
constexpr size_t kOffCostA = kOffPlaneB + al(kPx * 16);
constexpr size_t kOffCostB = kOffCostA + al(kPx * 4);
constexpr size_t kTotal = kOffCostB + al(kPx * 4);
static_assert(kTotal == RCMVS_NOALLOC_SCRATCH_BYTES, "header constant out of date");
static_assert(al(sizeof(DevView) * kViews) + al(sizeof(int32_t) * (kViews + 1)) + al(sizeof(double) * 4 * kViews) +
                      al(sizeof(DevJob)) + al(2 * sizeof(int32_t)) <= kDesc,
              "descriptor region too small");

}  // namespace

// The scratch array.  Host code must not use this name as a device address:
// the set-up below asks the runtime for the address on the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[RCMVS_NOALLOC_SCRATCH_BYTES];

namespace {

// The array's device address on the current device.  Looked up on every
// call rather than cached: the lookup allocates nothing, and after a
// cudaDeviceReset the module is loaded again in a new context where the
// array may sit at another address.  The first lookup on a device loads the
// module there (reserving the array), which is why the first call on a
// device must not be made during a stream capture.
int scratch_for_current_device(void** out) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return RCMVS_E_CUDA;
    *out = p;
    return RCMVS_OK;
}

// Flags this entry point accepts: it always runs the one-launch-per-step
// schedule and never skips duplicate or repeated candidates (so
// NO_SKIP_DUPLICATES and NO_REPEAT_SKIP hold trivially); SEED_AND_SWEEP
// concerns the learned init only.
constexpr uint32_t kNoallocFlags = RCMVS_FLAG_ONE_CANDIDATE | RCMVS_FLAG_NO_SKIP_DUPLICATES | RCMVS_FLAG_INIT_ONLY |
                                   RCMVS_FLAG_SEED_AND_SWEEP | RCMVS_FLAG_NO_REPEAT_SKIP;

bool finite_pos(double x) { return x > 0.0 && x < 1e300; }

bool good_view(const rcmvs_view& v) {
    if (v.w <= 0 || v.h <= 0 || !v.gray) return false;
    if (!(v.f == v.f) || v.f == 0.0 || !(v.f > -1e300 && v.f < 1e300)) return false;
    const double s[] = {v.cx, v.cy, v.k, v.R[0], v.R[1], v.R[2], v.R[3], v.R[4], v.R[5], v.R[6], v.R[7], v.R[8],
                        v.t[0], v.t[1], v.t[2]};
    for (double x : s)
        if (!(x > -1e300 && x < 1e300)) return false;
    return true;
}

}  // namespace

extern "C" int rcmvs_estimate_depth_noalloc(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                                            const int32_t* srcs, int32_t n_src, double zmin, double zmax,
                                            const rcmvs_options* opts, float* depth_dev, float* cost_dev,
                                            void* stream) {
    if (!views || n_views <= 0 || ref_idx < 0 || ref_idx >= n_views || n_src < 0 || (n_src > 0 && !srcs) || !opts ||
        !depth_dev || !cost_dev || (opts->flags & ~kNoallocFlags) || opts->passes > RCMVS_MAX_PASSES)
        return RCMVS_E_ARG;
    if (!(finite_pos(zmin) && finite_pos(zmax))) return RCMVS_E_ARG;
    if (n_src > RCMVS_NOALLOC_MAX_SOURCES) return RCMVS_E_LIMIT;
    int local[kViews];
    local[0] = ref_idx;
    for (int s = 0; s < n_src; ++s) {
        if (srcs[s] < 0 || srcs[s] >= n_views) return RCMVS_E_ARG;
        local[1 + s] = srcs[s];
    }
    const int nv = 1 + n_src;
    for (int i = 0; i < nv; ++i) {
        const rcmvs_view& v = views[local[i]];
        if (!good_view(v)) return RCMVS_E_ARG;
        if ((uint32_t)(v.w > v.h ? v.w : v.h) > opts->max_dim) return RCMVS_E_ARG;
        if ((size_t)v.w * (size_t)v.h > kPx) return RCMVS_E_LIMIT;
    }
    const TileShape ts = default_tile_shape(opts);
    if (!tile_shape_ok(ts)) return RCMVS_E_ARG;

    void* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    unsigned char* B = (unsigned char*)base;
    cudaStream_t st = (cudaStream_t)stream;

    // ---- descriptors, built on the stack
    DevView dv[kViews];
    int32_t tile_start[kViews + 1];
    double cams[4 * kViews];
    int tiles = 0;
    for (int i = 0; i < nv; ++i) {
        const rcmvs_view& v = views[local[i]];
        dv[i] = DevView{v.w, v.h, (int64_t)(i * kPx)};
        tile_start[i] = tiles;
        tiles += census_tiles(v.w, v.h);
        cams[4 * i] = v.f;
        cams[4 * i + 1] = v.cx;
        cams[4 * i + 2] = v.cy;
        cams[4 * i + 3] = v.k;
    }
    tile_start[nv] = tiles;

    // the job: mvs/src/stereo.rs:114-151 (f64 relative poses cast to f32)
    DevJob J;  // 2.6 KB on the stack: no heap allocation
    std::memset(&J, 0, sizeof(J));
    const rcmvs_view& r = views[ref_idx];
    J.view = 0;
    J.nsrc = n_src;
    J.w = r.w;
    J.h = r.h;
    J.off = 0;
    J.zmin = (float)zmin;
    J.zmax = (float)zmax;
    J.inv_min = 1.0f / J.zmax;
    J.inv_max = 1.0f / J.zmin;
    J.tiles_x = (r.w + ts.tw - 1) / ts.tw;
    J.tiles_y = (r.h + ts.th - 1) / ts.th;
    J.tiles = J.tiles_x * J.tiles_y;
    J.tile_base = 0;
    J.tw = ts.tw;
    J.th = ts.th;
    for (int s = 0; s < n_src; ++s) {
        const rcmvs_view& sv = views[srcs[s]];
        DevSrc& D = J.src[s];
        double rs64[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                rs64[3 * i + j] = sv.R[3 * i] * r.R[3 * j] + sv.R[3 * i + 1] * r.R[3 * j + 1] + sv.R[3 * i + 2] * r.R[3 * j + 2];
        for (int i = 0; i < 9; ++i) D.rs[i] = (float)rs64[i];
        for (int i = 0; i < 3; ++i) {
            double rt = rs64[3 * i] * r.t[0] + rs64[3 * i + 1] * r.t[1] + rs64[3 * i + 2] * r.t[2];
            D.ts[i] = (float)(sv.t[i] - rt);
        }
        D.f = (float)sv.f;
        D.cx = (float)sv.cx;
        D.cy = (float)sv.cy;
        D.k = (float)sv.k;
        D.w = sv.w;
        D.h = sv.h;
        D.off = (int64_t)((1 + s) * kPx);
    }
    int32_t job_start[2] = {0, J.tiles};

    unsigned char* d = B;
    DevView* d_views = (DevView*)d;
    d += al(sizeof(dv));
    int32_t* d_tile_start = (int32_t*)d;
    d += al(sizeof(tile_start));
    double* d_cams = (double*)d;
    d += al(sizeof(cams));
    DevJob* d_job = (DevJob*)d;
    d += al(sizeof(DevJob));
    int32_t* d_job_start = (int32_t*)d;
    uint8_t* gray = B + kOffGray;
    uint64_t* census = (uint64_t*)(B + kOffCensus);
    float2* rays = (float2*)(B + kOffRays);
    PlaneBuf A{(float4*)(B + kOffPlaneA), (float*)(B + kOffCostA)};
    PlaneBuf Bp{(float4*)(B + kOffPlaneB), (float*)(B + kOffCostB)};

#define NCK(x)                                   \
    do {                                         \
        if ((x) != cudaSuccess) return RCMVS_E_CUDA; \
    } while (0)
    // pageable -> device copies return once the source has been staged, so
    // the stack buffers above may go out of scope afterwards
    NCK(cudaMemcpyAsync(d_views, dv, sizeof(DevView) * nv, cudaMemcpyHostToDevice, st));
    NCK(cudaMemcpyAsync(d_tile_start, tile_start, sizeof(int32_t) * (nv + 1), cudaMemcpyHostToDevice, st));
    NCK(cudaMemcpyAsync(d_cams, cams, sizeof(double) * 4 * nv, cudaMemcpyHostToDevice, st));
    NCK(cudaMemcpyAsync(d_job, &J, sizeof(DevJob), cudaMemcpyHostToDevice, st));
    NCK(cudaMemcpyAsync(d_job_start, job_start, sizeof(job_start), cudaMemcpyHostToDevice, st));
    for (int i = 0; i < nv; ++i) {
        const rcmvs_view& v = views[local[i]];
        NCK(cudaMemcpyAsync(gray + i * kPx, v.gray, (size_t)v.w * v.h, cudaMemcpyDeviceToDevice, st));
    }
    NCK(launch_census_rays(d_views, d_tile_start, nv, tiles, gray, census, rays, d_cams, st));
    const int nh = (int)(opts->num_hyp > 2u ? opts->num_hyp : 2u);
    const int variant = (opts->flags & RCMVS_FLAG_ONE_CANDIDATE) ? 1 : 0;
    const LaunchGeom g{ts.tw * ts.th, stereo_smem_bytes(ts), J.tiles, nullptr};
    NCK(launch_init(d_job, d_job_start, 1, g, nh, census, rays, A, nullptr, st, variant));
    const uint64_t n_passes = rcmvs_pass_count(opts);
    for (uint64_t pass = 0; pass < n_passes; ++pass) {
        const float t = (float)pass / (float)n_passes;  // stereo.rs:275-277
        const float sig_inv = 0.02f * powf(0.28f, t * 4.0f);
        const float sig_n = 0.30f * powf(0.42f, t * 4.0f);
        NCK(launch_pass(d_job, d_job_start, 1, g, pass, sig_inv, sig_n, census, rays, A, Bp, nullptr, st));
        PlaneBuf tmp = A;
        A = Bp;
        Bp = tmp;
    }
    NCK(launch_gate(d_job, d_job_start, 1, g, opts->cost_thr, census, A, depth_dev, cost_dev, nullptr, st));
#undef NCK
    return RCMVS_OK;
}
