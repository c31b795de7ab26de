// match.cu — SIFT descriptor matching on sm_100a.
//
// Restates sfm-lite/src/matching.rs:22-95 (match_pair) for a batch of image
// pairs: for every descriptor of A the nearest and second-nearest descriptor
// of B by squared L2 distance, the same from B to A, Lowe's ratio test both
// ways and the mutual-best check.
//
// The reference sums (a_k - b_k)^2 serially over k = 0..127 in f32.  A GEMM
// (2 - 2 a.b) would round differently and move ratio-test and tie decisions,
// so the distances are computed as written, on the FP32 pipes:
//
//   dist_kernel   64x64 distances per block, 4x4 per thread; 32-wide k chunks
//                 of both tiles staged k-major in shared memory (float4 reads,
//                 conflict-free), each distance accumulated in k order; with
//                 --fmad=false every difference, square and sum rounds as in
//                 the reference.  The distances never leave the block: it
//                 writes, for each of its rows and columns, the (best, index,
//                 second) over the tile, merged through shuffles and shared
//                 memory.  One distance serves both directions: (a - b)^2 and
//                 the reference's backward (a - b)^2 are the same number.
//   rows_kernel   one thread per row: the tiles' partials merged by value
//   cols_kernel   with the lower index winning ties -- the first minimum and
//                 the second smallest value, exactly what the reference's
//                 sequential scan keeps (the merge is associative, so the
//                 order of the tiles does not matter)
//   decide_kernel the reference's tests per row of A
//
// Pairs run in chunks whose tile partials (the per-tile best/second entries
// of every row and column, 12 bytes each; no distance matrix is written)
// fit P_BUDGET; results come back as per-pair lists in the reference's order
// (ascending index in A).
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ctx_internal.cuh"

namespace rcmvs {

namespace {

constexpr int DESC_LEN = 128;
constexpr int TILE = 64;
constexpr int KC = 32;
constexpr size_t P_BUDGET = size_t(1) << 28;  // bytes of tile partials per chunk

struct PairJob {
    int64_t a_off, b_off;      // first descriptor of each frame (in descriptors)
    int64_t prow_off, pcol_off;  // tile partials: [column tile][na] rows, [row tile][nb] columns
    int32_t na, nb;
    int32_t row_off, col_off;  // into the chunk's forward / backward results
};

struct Nearest {
    uint32_t idx;
    float d1, d2;
};

// Sequential-scan state: the first minimum and the second smallest value.
__device__ __forceinline__ void push(float s, uint32_t j, float& best, uint32_t& bi, float& second) {
    if (s < best) {
        second = best;
        best = s;
        bi = j;
    } else if (s < second) {
        second = s;
    }
}

// The same state of a union of two disjoint parts: the smaller best (the
// lower index among equal values) and the second smallest value of the union.
__device__ __forceinline__ void merge(float& best, uint32_t& bi, float& second, float ob, uint32_t oi, float os) {
    const float nsec = fminf(fmaxf(best, ob), fminf(second, os));
    if (ob < best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
    }
    second = nsec;
}

__global__ void __launch_bounds__(256) dist_kernel(const float* __restrict__ desc, const PairJob* __restrict__ jobs,
                                                   Nearest* __restrict__ rowpart, Nearest* __restrict__ colpart) {
    __shared__ __align__(16) float As[KC][TILE];
    __shared__ __align__(16) float Bs[KC][TILE];
    __shared__ Nearest cpart[8][TILE];
    const PairJob J = jobs[blockIdx.z];
    const int r0 = blockIdx.y * TILE, c0 = blockIdx.x * TILE;
    if (r0 >= J.na || c0 >= J.nb) return;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const float* A = desc + J.a_off * DESC_LEN;
    const float* B = desc + J.b_off * DESC_LEN;
    float acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;
    for (int k0 = 0; k0 < DESC_LEN; k0 += KC) {
        // 64 rows x 8 float4 per tile; a warp covers 32 rows of one float4
        for (int e = threadIdx.x; e < TILE * (KC / 4); e += 256) {
            const int row = e % TILE, q = e / TILE;
            float4 va = make_float4(0.f, 0.f, 0.f, 0.f), vb = va;
            if (r0 + row < J.na) va = *reinterpret_cast<const float4*>(A + (int64_t)(r0 + row) * DESC_LEN + k0 + 4 * q);
            if (c0 + row < J.nb) vb = *reinterpret_cast<const float4*>(B + (int64_t)(c0 + row) * DESC_LEN + k0 + 4 * q);
            As[4 * q][row] = va.x;
            As[4 * q + 1][row] = va.y;
            As[4 * q + 2][row] = va.z;
            As[4 * q + 3][row] = va.w;
            Bs[4 * q][row] = vb.x;
            Bs[4 * q + 1][row] = vb.y;
            Bs[4 * q + 2][row] = vb.z;
            Bs[4 * q + 3][row] = vb.w;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < KC; ++kk) {
            const float4 a4 = *reinterpret_cast<const float4*>(&As[kk][ty * 4]);
            const float4 b4 = *reinterpret_cast<const float4*>(&Bs[kk][tx * 4]);
            const float a[4] = {a4.x, a4.y, a4.z, a4.w};
            const float b[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float d = a[r] - b[c];
                    acc[r][c] = acc[r][c] + d * d;
                }
        }
        __syncthreads();
    }
    // Rows: each of this thread's 4 rows over its 4 columns, then over the
    // 16 threads of the row group (lanes 0-15 or 16-31 of the warp).
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int ia = r0 + ty * 4 + r;
        float best = INFINITY, second = INFINITY;
        uint32_t bi = UINT32_MAX;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int ib = c0 + tx * 4 + c;
            if (ia < J.na && ib < J.nb) push(acc[r][c], (uint32_t)ib, best, bi, second);
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1)
            merge(best, bi, second, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, bi, o),
                  __shfl_xor_sync(0xffffffffu, second, o));
        if (tx == 0 && ia < J.na) rowpart[J.prow_off + (int64_t)blockIdx.x * J.na + ia] = Nearest{bi, best, second};
    }
    // Columns: each of this thread's 4 columns over its 4 rows, then the two
    // row groups of the warp, then the 8 warps through shared memory.
    const int wid = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int ib = c0 + tx * 4 + c;
        float best = INFINITY, second = INFINITY;
        uint32_t bi = UINT32_MAX;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int ia = r0 + ty * 4 + r;
            if (ia < J.na && ib < J.nb) push(acc[r][c], (uint32_t)ia, best, bi, second);
        }
        merge(best, bi, second, __shfl_xor_sync(0xffffffffu, best, 16), __shfl_xor_sync(0xffffffffu, bi, 16),
              __shfl_xor_sync(0xffffffffu, second, 16));
        if ((threadIdx.x & 16) == 0) cpart[wid][tx * 4 + c] = Nearest{bi, best, second};
    }
    __syncthreads();
    if (threadIdx.x < TILE) {
        const int ib = c0 + threadIdx.x;
        Nearest m = cpart[0][threadIdx.x];
        for (int q = 1; q < 8; ++q) {
            const Nearest o = cpart[q][threadIdx.x];
            merge(m.d1, m.idx, m.d2, o.d1, o.idx, o.d2);
        }
        if (ib < J.nb) colpart[J.pcol_off + (int64_t)blockIdx.y * J.nb + ib] = m;
    }
}

// The tiles' partials of each row (over column tiles) and of each column
// (over row tiles), merged into the nearest and second-nearest of the row or
// column; one thread each.
__global__ void __launch_bounds__(256) rows_kernel(const PairJob* __restrict__ jobs, const Nearest* __restrict__ rowpart,
                                                   Nearest* __restrict__ fwd) {
    const PairJob J = jobs[blockIdx.y];
    const int ia = blockIdx.x * 256 + threadIdx.x;
    if (ia >= J.na) return;
    const int nct = (J.nb + TILE - 1) / TILE;
    Nearest m{UINT32_MAX, INFINITY, INFINITY};
    for (int t = 0; t < nct; ++t) {
        const Nearest o = rowpart[J.prow_off + (int64_t)t * J.na + ia];
        merge(m.d1, m.idx, m.d2, o.d1, o.idx, o.d2);
    }
    fwd[J.row_off + ia] = m;
}

__global__ void __launch_bounds__(256) cols_kernel(const PairJob* __restrict__ jobs, const Nearest* __restrict__ colpart,
                                                   Nearest* __restrict__ bwd) {
    const PairJob J = jobs[blockIdx.y];
    const int ib = blockIdx.x * 256 + threadIdx.x;
    if (ib >= J.nb) return;
    const int nrt = (J.na + TILE - 1) / TILE;
    Nearest m{UINT32_MAX, INFINITY, INFINITY};
    for (int t = 0; t < nrt; ++t) {
        const Nearest o = colpart[J.pcol_off + (int64_t)t * J.nb + ib];
        merge(m.d1, m.idx, m.d2, o.d1, o.idx, o.d2);
    }
    bwd[J.col_off + ib] = m;
}

// matching.rs:74-94
__global__ void decide_kernel(const PairJob* __restrict__ jobs, const Nearest* __restrict__ fwd,
                              const Nearest* __restrict__ bwd, float ratio, uint32_t* __restrict__ match_b) {
    const PairJob J = jobs[blockIdx.y];
    const int ia = blockIdx.x * 256 + threadIdx.x;
    if (ia >= J.na) return;
    uint32_t out = UINT32_MAX;
    const Nearest f = fwd[J.row_off + ia];
    if (f.idx != UINT32_MAX && isfinite(f.d2) && !(f.d1 > 0.9f || f.d1 > ratio * f.d2)) {
        const Nearest g = bwd[J.col_off + f.idx];
        if (g.idx == (uint32_t)ia && isfinite(g.d2) && !(g.d1 > ratio * g.d2)) out = f.idx;
    }
    match_b[J.row_off + ia] = out;
}

int mfail(rcmvs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

#define MCK(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return mfail(ctx, e_ == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,    \
                         std::string(#x) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

// Context arena slots 160-167.
enum { M_DESC = 160, M_JOBS, M_ROWP, M_FWD, M_BWD, M_MB, M_COLP };

}  // namespace
}  // namespace rcmvs

using namespace rcmvs;

extern "C" {

void rcmvs_matches_free(rcmvs_matches* m) {
    if (!m) return;
    std::free(m->offsets);
    std::free(m->a);
    std::free(m->b);
    m->offsets = nullptr;
    m->a = m->b = nullptr;
    m->n_pairs = 0;
}

static int match_pairs_impl(rcmvs_ctx* ctx, const float* const* desc, const int32_t* n_desc, int32_t n_frames,
                            const int32_t* pairs, int32_t n_pairs, double ratio, rcmvs_matches* out);

int rcmvs_match_pairs(rcmvs_ctx* ctx, const float* const* desc, const int32_t* n_desc, int32_t n_frames,
                      const int32_t* pairs, int32_t n_pairs, double ratio, rcmvs_matches* out) {
    if (!ctx || !out || n_frames < 0 || n_pairs < 0 || (n_frames > 0 && (!desc || !n_desc)) ||
        (n_pairs > 0 && !pairs))
        return mfail(ctx, RCMVS_E_ARG, "rcmvs_match_pairs: bad argument");
    std::memset(out, 0, sizeof(*out));
    const int rc = match_pairs_impl(ctx, desc, n_desc, n_frames, pairs, n_pairs, ratio, out);
    if (rc) rcmvs_matches_free(out);  // nothing half-built reaches the caller
    return rc;
}

static int match_pairs_impl(rcmvs_ctx* ctx, const float* const* desc, const int32_t* n_desc, int32_t n_frames,
                            const int32_t* pairs, int32_t n_pairs, double ratio, rcmvs_matches* out) {
    std::vector<int64_t> foff(n_frames + 1, 0);
    for (int f = 0; f < n_frames; ++f) {
        if (n_desc[f] < 0 || (n_desc[f] > 0 && !desc[f])) return mfail(ctx, RCMVS_E_ARG, "bad descriptor set");
        foff[f + 1] = foff[f] + n_desc[f];
    }
    for (int p = 0; p < n_pairs; ++p)
        if (pairs[2 * p] < 0 || pairs[2 * p] >= n_frames || pairs[2 * p + 1] < 0 || pairs[2 * p + 1] >= n_frames)
            return mfail(ctx, RCMVS_E_ARG, "pair names a frame out of range");
    out->n_pairs = (uint64_t)n_pairs;
    out->offsets = (uint64_t*)std::calloc((size_t)n_pairs + 1, sizeof(uint64_t));
    if (!out->offsets) return mfail(ctx, RCMVS_E_NOMEM, "host allocation failed");
    std::vector<uint32_t> ra, rb;
    MCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    DeviceArena& A = ctx->arena;
    void* p_desc;
    MCK(A.get(M_DESC, sizeof(float) * DESC_LEN * (size_t)std::max<int64_t>(foff[n_frames], 1), &p_desc));
    for (int f = 0; f < n_frames; ++f)
        if (n_desc[f] > 0)
            MCK(cudaMemcpyAsync((float*)p_desc + foff[f] * DESC_LEN, desc[f], sizeof(float) * DESC_LEN * n_desc[f],
                                cudaMemcpyHostToDevice, st));
    const float r32 = (float)ratio;
    int p = 0;
    while (p < n_pairs) {
        // a chunk of pairs whose distance matrices fit the budget (at least one)
        std::vector<PairJob> jobs;
        int64_t prow = 0, pcol = 0, rows = 0, cols = 0;
        int max_na = 0, max_nb = 0;
        while (p < n_pairs && jobs.size() < 65535) {
            const int fa = pairs[2 * p], fb = pairs[2 * p + 1];
            const int na = n_desc[fa], nb = n_desc[fb];
            const int64_t pr = (int64_t)((nb + TILE - 1) / TILE) * na, pc = (int64_t)((na + TILE - 1) / TILE) * nb;
            if (!jobs.empty() && (size_t)(prow + pr + pcol + pc) * sizeof(Nearest) > P_BUDGET) break;
            jobs.push_back(PairJob{foff[fa], foff[fb], prow, pcol, na, nb, (int32_t)rows, (int32_t)cols});
            prow += pr;
            pcol += pc;
            rows += na;
            cols += nb;
            max_na = std::max(max_na, na);
            max_nb = std::max(max_nb, nb);
            ++p;
            if (rows > INT32_MAX / 2 || cols > INT32_MAX / 2) break;
        }
        const int first = p - (int)jobs.size();
        if (max_na > 0 && max_nb > 0) {
            void *p_jobs, *p_rowp, *p_colp, *p_fwd, *p_bwd, *p_mb;
            MCK(A.get(M_JOBS, sizeof(PairJob) * jobs.size(), &p_jobs));
            MCK(A.get(M_ROWP, sizeof(Nearest) * (size_t)std::max<int64_t>(prow, 1), &p_rowp));
            MCK(A.get(M_COLP, sizeof(Nearest) * (size_t)std::max<int64_t>(pcol, 1), &p_colp));
            MCK(A.get(M_FWD, sizeof(Nearest) * (size_t)rows, &p_fwd));
            MCK(A.get(M_BWD, sizeof(Nearest) * (size_t)cols, &p_bwd));
            MCK(A.get(M_MB, sizeof(uint32_t) * (size_t)rows, &p_mb));
            MCK(cudaMemcpyAsync(p_jobs, jobs.data(), sizeof(PairJob) * jobs.size(), cudaMemcpyHostToDevice, st));
            const unsigned nj = (unsigned)jobs.size();
            const SpanHook& hook = ctx->hook();
            hook.begin("match_dist");
            dist_kernel<<<dim3((max_nb + TILE - 1) / TILE, (max_na + TILE - 1) / TILE, nj), 256, 0, st>>>(
                (const float*)p_desc, (const PairJob*)p_jobs, (Nearest*)p_rowp, (Nearest*)p_colp);
            MCK(cudaGetLastError());
            hook.end("match_dist");
            hook.begin("match_select");
            rows_kernel<<<dim3((max_na + 255) / 256, nj), 256, 0, st>>>((const PairJob*)p_jobs,
                                                                       (const Nearest*)p_rowp, (Nearest*)p_fwd);
            MCK(cudaGetLastError());
            cols_kernel<<<dim3((max_nb + 255) / 256, nj), 256, 0, st>>>((const PairJob*)p_jobs,
                                                                       (const Nearest*)p_colp, (Nearest*)p_bwd);
            MCK(cudaGetLastError());
            decide_kernel<<<dim3((max_na + 255) / 256, nj), 256, 0, st>>>(
                (const PairJob*)p_jobs, (const Nearest*)p_fwd, (const Nearest*)p_bwd, r32, (uint32_t*)p_mb);
            MCK(cudaGetLastError());
            hook.end("match_select");
            std::vector<uint32_t> mb((size_t)rows);
            MCK(cudaMemcpyAsync(mb.data(), p_mb, sizeof(uint32_t) * rows, cudaMemcpyDeviceToHost, st));
            MCK(cudaStreamSynchronize(st));
            for (size_t c = 0; c < jobs.size(); ++c) {
                for (int ia = 0; ia < jobs[c].na; ++ia) {
                    const uint32_t b = mb[(size_t)jobs[c].row_off + ia];
                    if (b != UINT32_MAX) {
                        ra.push_back((uint32_t)ia);
                        rb.push_back(b);
                    }
                }
                out->offsets[first + c + 1] = ra.size();
            }
        } else {
            for (size_t c = 0; c < jobs.size(); ++c) out->offsets[first + c + 1] = ra.size();
        }
    }
    const size_t n = ra.size();
    out->a = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<size_t>(n, 1));
    out->b = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<size_t>(n, 1));
    if (!out->a || !out->b) {
        rcmvs_matches_free(out);
        return mfail(ctx, RCMVS_E_NOMEM, "host allocation failed");
    }
    if (n) {
        std::memcpy(out->a, ra.data(), sizeof(uint32_t) * n);
        std::memcpy(out->b, rb.data(), sizeof(uint32_t) * n);
    }
    return RCMVS_OK;
}

}  // extern "C"
