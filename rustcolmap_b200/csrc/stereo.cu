// stereo.cu — census patch-match stereo on sm_100a.
//
// Restates mvs/src/stereo.rs:
//   plane_cost      stereo.rs:158-228   (device function plane_cost)
//   init sweep      stereo.rs:247-269   (init_kernel)
//   Jacobi passes   stereo.rs:271-371   (pass_kernel, one launch per pass)
//   texture gate    stereo.rs:373-393   (gate_kernel)
//   pixel RNG       stereo.rs:47-78
//
// Bit-exactness: the library is compiled with --fmad=false and IEEE divide
// and square root, and every f32 expression keeps the reference's operand
// order, so each pixel's cost, abort decision, RNG draw and accepted plane is
// identical to the CPU code.  The f32 sum of the 25*K window terms stays a
// serial per-thread chain in (source, dy, dx) order because the early-abort
// test reads its partial values.
//
// Layout: one thread per reference pixel; one block per TW x TH tile of one
// job (all jobs of a batch in one launch).  The block stages its jobs'
// support-view parameters, a 49-entry h/48 table, and the tile's rays and
// census with a 2-pixel clamped halo in shared memory; support-view census
// words are gathered through the read-only path (L1/L2).
#include <algorithm>
#include <climits>

#include "rcmvs_internal.cuh"
#include "learned.cuh"

namespace rcmvs {

namespace {

constexpr int HALO = 2;  // 5x5 window (stereo.rs:41)

__device__ __forceinline__ int find_item(const int32_t* start, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------- RNG
// stereo.rs:47-57
__device__ __forceinline__ uint64_t pixel_rng(int32_t x, int32_t y, uint64_t salt) {
    uint64_t s = ((uint64_t)(int64_t)x * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)(int64_t)y * 0xC2B2AE3D27D4EB4Full) ^
                 (salt * 0x165667B19E3779F9ull);
    s ^= s >> 30;
    s *= 0xBF58476D1CE4E5B9ull;
    s ^= s >> 27;
    s *= 0x94D049BB133111EBull;
    return s ^ (s >> 31);
}
// stereo.rs:59-78.  (x>>40) < 2^24 converts exactly; the divide by 2^24 is
// an exact power-of-two scale, written as a multiply.
__device__ __forceinline__ float uniform01(uint64_t& s) {
    uint64_t x = s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    s = x;
    return (float)(x >> 40) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ float gauss3(uint64_t& s) {
    float a = uniform01(s);
    float b = uniform01(s);
    float c = uniform01(s);
    return a + b + c - 1.5f;
}

// ---------------------------------------------------------------- tile setup
struct Tile {
    const DevJob* job;
    int x0, y0;
    int tw, th;  // the job's tile shape
    int stw;     // shared tile row pitch (tw + 2*HALO)
};

struct Smem {
    DevSrc* src;     // RCMVS_MAX_SOURCES
    float* tab;      // 64 (49 used): h / 48.0f
    float2* ray;     // (th+4)*(tw+4)
    uint64_t* cen;   // (th+4)*(tw+4)
};

__host__ __device__ inline size_t smem_bytes(int tw, int th) {
    size_t cells = (size_t)(tw + 2 * HALO) * (th + 2 * HALO);
    return sizeof(DevSrc) * RCMVS_MAX_SOURCES + 64 * sizeof(float) + cells * sizeof(float2) +
           cells * sizeof(uint64_t);
}

__device__ __forceinline__ Smem carve(unsigned char* base, int tw, int th) {
    Smem s;
    size_t cells = (size_t)(tw + 2 * HALO) * (th + 2 * HALO);
    s.src = reinterpret_cast<DevSrc*>(base);
    s.tab = reinterpret_cast<float*>(base + sizeof(DevSrc) * RCMVS_MAX_SOURCES);
    s.ray = reinterpret_cast<float2*>(s.tab + 64);
    s.cen = reinterpret_cast<uint64_t*>(s.ray + cells);
    return s;
}

// Tile scheduler of the persistent (PERSIST) stereo kernels; all threads of
// the block call it and get the same answer.  The block takes tile after
// tile from `queue` (a counter zeroed before the launch) until every tile of
// the launch has been handed out: the (view, tile) work queue.  Returns -1
// when the block is done.  Non-persistent kernels compute tile blockIdx.x
// once.
__device__ __forceinline__ int next_tile(unsigned int* queue, int tiles, int it, int* s_tile) {
    if (it > 0) __syncthreads();  // the previous tile's shared data is no longer read
    if (threadIdx.x == 0) *s_tile = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int t = *s_tile;
    return t < tiles ? t : -1;
}

// Resolves launch tile `tile` to its job, carves shared memory for the job's
// tile shape and stages the job's sources, the h/48 table and the halo tile.
// All threads call it (threads past the job's tw*th pixels help load).
__device__ __forceinline__ void load_tile(const DevJob* jobs, const int32_t* job_start, int n_jobs, int tile,
                                          const uint64_t* __restrict__ census, const float2* __restrict__ rays,
                                          unsigned char* smem_raw, Smem& sm, Tile& T) {
    const int j = find_item(job_start, n_jobs, tile);
    const DevJob* J = jobs + j;
    T.job = J;
    const int tw = J->tw, th = J->th;
    T.tw = tw;
    T.th = th;
    const int t = tile - job_start[j];
    const int tiles_x = J->tiles_x;
    T.x0 = (t % tiles_x) * tw;
    T.y0 = (t / tiles_x) * th;
    T.stw = tw + 2 * HALO;
    sm = carve(smem_raw, tw, th);
    const int nthr = blockDim.x;
    {
        const int nwords = J->nsrc * (int)(sizeof(DevSrc) / 4);
        const uint32_t* srcw = reinterpret_cast<const uint32_t*>(J->src);
        uint32_t* dstw = reinterpret_cast<uint32_t*>(sm.src);
        for (int i = threadIdx.x; i < nwords; i += nthr) dstw[i] = srcw[i];
    }
    for (int h = threadIdx.x; h < 49; h += nthr) sm.tab[h] = (float)h / 48.0f;
    const int w = J->w, hgt = J->h;
    const int cells = (tw + 2 * HALO) * (th + 2 * HALO);
    const size_t off = (size_t)J->off;
    for (int i = threadIdx.x; i < cells; i += nthr) {
        int sx = i % T.stw, sy = i / T.stw;
        int gx = min(max(T.x0 - HALO + sx, 0), w - 1);
        int gy = min(max(T.y0 - HALO + sy, 0), hgt - 1);
        size_t g = off + (size_t)gy * w + gx;
        sm.ray[i] = __ldg(rays + g);
        sm.cen[i] = __ldg(census + g);
    }
    __syncthreads();
}

struct WorkCount {
    unsigned long long evals, rows;
};

// Early rejection (exact): a candidate is kept only if its cost is strictly
// below best_c, and the window sum only grows (each term adds a
// non-negative h/48, and f32 addition of a non-negative value never lowers
// the sum), so once sum >= best_c * total the final cost sum_final / total
// is >= best_c and the candidate cannot be kept: the evaluation may stop.
// The bound is rounded up by one ulp so that the f32 product's rounding can
// never make the test fire early.  Skipping such a candidate changes no
// state -- best_c and the kept plane are only updated by a kept candidate,
// and no RNG draw depends on a cost -- so every output bit is the
// reference's; only the work counters see fewer rows.  +inf disables it
// (best_c = +inf before the first hypothesis, and the reference call
// sequence of RCMVS_FLAG_NO_SKIP_DUPLICATES).
__device__ __forceinline__ float reject_bound(float best_c, float total) {
    const float t = best_c * total;
    return t < INFINITY ? __int_as_float(__float_as_int(t) + 1) : INFINITY;
}

// Denominator of the abort test after window row dy of support view si
// (stereo.rs:215-221): rows_done * 5 * (si + 1), exact in f32.  With `ahead`
// (an exact shortcut, off for the reference's call sequence) it is capped at
// 5 * (si + 2), the denominator of the test after the first row of the next
// view.  The window sum never decreases (every term adds h/48 >= 0) and
// sum / den only grows as den falls, so once sum / (5 * (si + 2)) exceeds the
// threshold that later test is certain to fire (if none before it does):
// the evaluation's result, the abort value, is already known.
__device__ __forceinline__ float abort_den(int dy, int si, int nsrc, bool ahead) {
    const float den = (float)(dy + 1) * 5.0f * (float)(si + 1);
    return (ahead && si + 1 < nsrc) ? fminf(den, 5.0f * (float)(si + 2)) : den;
}

// ---------------------------------------------------------------- plane_cost
// One support view in registers.
struct SrcRegs {
    float rs0, rs1, rs2, rs3, rs4, rs5, rs6, rs7, rs8, ts0, ts1, ts2, f, cx, cy, k;
    int sw, sh;
    float swf, shf;  // sw, sh as floats (exact: sizes < 2^23)
    const uint64_t* __restrict__ sc;
};

__device__ __forceinline__ SrcRegs load_src(const DevSrc& s, const uint64_t* __restrict__ census) {
    SrcRegs r;
    r.rs0 = s.rs[0];
    r.rs1 = s.rs[1];
    r.rs2 = s.rs[2];
    r.rs3 = s.rs[3];
    r.rs4 = s.rs[4];
    r.rs5 = s.rs[5];
    r.rs6 = s.rs[6];
    r.rs7 = s.rs[7];
    r.rs8 = s.rs[8];
    r.ts0 = s.ts[0];
    r.ts1 = s.ts[1];
    r.ts2 = s.ts[2];
    r.f = s.f;
    r.cx = s.cx;
    r.cy = s.cy;
    r.k = s.k;
    r.sw = s.w;
    r.sh = s.h;
    r.swf = (float)s.w;
    r.shf = (float)s.h;
    r.sc = census + s.off;
    return r;
}

// Rust's `x as i32` (truncation toward zero, saturating, NaN -> 0) followed
// by the test 0 <= i < n (stereo.rs:204-210), without a conversion
// instruction: trunc(x) lies in [0, n) exactly when x > -1 and x < n, NaN
// included (it converts to 0).  The index is trunc(max(x, 0)), formed
// exactly by adding 2^23 with rounding toward zero (valid for x < n <= 2^23,
// where the sum's spacing is 1) and reading the integer off the mantissa.
// `nf` is n as a float.
__device__ __forceinline__ bool trunc_index(float x, float nf, int& i) {
    i = __float_as_int(__fadd_rz(fmaxf(x, 0.0f), 8388608.0f)) - 0x4B000000;
    return !(x <= -1.0f) && !(x >= nf);
}

// The five window terms of one row of one support view (stereo.rs:181-214),
// added to `sum` in dx order, with IEEE divides.  `row`: shared-tile index of
// the row's first window cell.  FRONTO: n = (0,0,1); then denom =
// 0*xo + 0*yo + 1 is exactly 1.0 for the finite rays the host admits, so
// z = d/1 = d, and both are skipped.
template <bool FRONTO, bool HSUM>
__device__ __forceinline__ float cost_row(const Smem& sm, int row, const SrcRegs& s, float nx, float ny, float nz,
                                          float d, float sum, int32_t& hs) {
    // Branch-free: every term's geometry is computed (a skipped term's
    // values are discarded), the gather reads a safe address when the term
    // is out, and the five h values are then added in dx order -- the same
    // f32 chain as the reference's, with the five terms free to overlap.
    int h[5];
#pragma unroll
    for (int dx = 0; dx < 5; ++dx) {
        const float2 r = sm.ray[row + dx];
        const float denom = FRONTO ? 1.0f : nx * r.x + ny * r.y + nz;
        const float z = FRONTO ? d : d / denom;
        const float xr = z * r.x;
        const float yr = z * r.y;
        const float xs = s.rs0 * xr + s.rs1 * yr + s.rs2 * z + s.ts0;
        const float ys = s.rs3 * xr + s.rs4 * yr + s.rs5 * z + s.ts1;
        const float zs = s.rs6 * xr + s.rs7 * yr + s.rs8 * z + s.ts2;
        const float xn = xs / zs;
        const float yn = ys / zs;
        const float dist = 1.0f + s.k * (xn * xn + yn * yn);
        int u, v;
        const bool in_u = trunc_index(s.f * xn * dist + s.cx, s.swf, u);
        const bool in_v = trunc_index(s.f * yn * dist + s.cy, s.shf, v);
        // stereo.rs:187-191 (denom), :196-201 (zs), :202-210 (bounds)
        const bool ok = !(denom < 0.05f) && !(zs < 1e-3f) && in_u && in_v;
        const uint64_t cs = __ldg(s.sc + (ok ? (size_t)v * s.sw + u : (size_t)0));
        const int hv = __popcll(sm.cen[row + dx] ^ cs);
        h[dx] = ok ? hv : 48;  // an excluded term adds 1.0 = tab[48]
    }
#pragma unroll
    for (int dx = 0; dx < 5; ++dx) {
        sum += sm.tab[h[dx]];
        if (HSUM) hs += h[dx];
    }
    return sum;
}

// stereo.rs:158-228, one candidate at a time.  (lx, ly): the pixel's
// position in the tile; window cell (dx, dy) of the pixel is shared cell
// (ly+dy)*stw + lx+dx (dx, dy in 0..4), which holds the clamped pixel
// (stereo.rs:179-184).
template <bool FRONTO, bool COUNT, bool HSUM>
__device__ __forceinline__ float plane_cost(const Smem& sm, int stw, int lx, int ly, int nsrc,
                                            const uint64_t* __restrict__ census, float nx, float ny, float nz,
                                            float d, float hint, float total, WorkCount& wc, int32_t* hsum,
                                            float rej = INFINITY, bool ahead = false) {
    float sum = 0.f;
    int32_t hs = 0;
    const float thr = hint + 0.12f;
    if (COUNT) wc.evals++;
    for (int si = 0; si < nsrc; ++si) {
        const SrcRegs s = load_src(sm.src[si], census);
        for (int dy = 0; dy < 5; ++dy) {
            sum = cost_row<FRONTO, HSUM>(sm, (ly + dy) * stw + lx, s, nx, ny, nz, d, sum, hs);
            if (COUNT) wc.rows++;
            if (sum / abort_den(dy, si, nsrc, ahead) > thr || sum >= rej) {
                if (HSUM) *hsum = hs;
                return 1e9f;
            }
        }
    }
    if (HSUM) *hsum = hs;
    return sum / total;
}

__device__ __forceinline__ void flush_work(const WorkCount& wc, unsigned long long* d_work) {
    unsigned long long e = wc.evals, r = wc.rows;
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_down_sync(0xffffffffu, e, o);
        r += __shfl_down_sync(0xffffffffu, r, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(d_work, e);
        atomicAdd(d_work + 1, r);
    }
}

// ---------------------------------------------------------------- init
// stereo.rs:247-269
template <bool COUNT, bool PERSIST>
__global__ void init_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start, int n_jobs,
                            int tiles, unsigned int* queue, int nh, const uint64_t* __restrict__ census,
                            const float2* __restrict__ rays, PlaneBuf out, unsigned long long* d_work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    WorkCount wc{0, 0};
    for (int it = 0; PERSIST || it == 0; ++it) {
        const int tile = PERSIST ? next_tile(queue, tiles, it, &s_tile) : (int)blockIdx.x;
        if (tile < 0) break;
        Smem sm;
        Tile T;
        load_tile(jobs, job_start, n_jobs, tile, census, rays, smem_raw, sm, T);
        const DevJob* J = T.job;
        const int lx = threadIdx.x % T.tw, ly = threadIdx.x / T.tw;
        const int x = T.x0 + lx, y = T.y0 + ly;
        if ((int)threadIdx.x < T.tw * T.th && x < J->w && y < J->h) {
            const int nsrc = J->nsrc;
            const float total = 5.0f * 5.0f * (float)nsrc;
            const float inv_min = J->inv_min, inv_max = J->inv_max;
            const bool early = out.d != nullptr;  // off for the reference call sequence
            float best_c = INFINITY;
            float best_d = 0.f;
            for (int hi = 0; hi < nh; ++hi) {
                const float inv = inv_min + (inv_max - inv_min) * (float)hi / (float)(nh - 1);
                const float d = 1.0f / inv;
                const float c = plane_cost<true, COUNT, false>(sm, T.stw, lx, ly, nsrc, census, 0.f, 0.f, 1.f, d,
                                                               best_c + 0.02f, total, wc, nullptr,
                                                               early ? reject_bound(best_c, total) : INFINITY, early);
                if (c < best_c) {
                    best_c = c;
                    best_d = d;
                }
            }
            const size_t i = (size_t)J->off + (size_t)y * J->w + x;
            out.nz[i] = make_float4(0.0f, 0.0f, 1.0f, best_d);
            out.cost[i] = fminf(best_c, 1.0f);
            if (out.d) out.d[i] = best_d;  // n = (0,0,1): d = z
        }
    }
    if (COUNT) flush_work(wc, d_work);
}

// ---------------------------------------------------------------- passes
// stereo.rs:274-371: one double-buffered pass.  Reads `prev` only, writes
// every pixel of `next` (the carried-over plane when nothing is accepted,
// which equals the reference's copy_from_slice at :278).
// Duplicate skip (with PlaneBuf::d): a neighbour's candidate whose normal
// and offset d equal, bit for bit, the plane the pixel's stored cost came
// from is not evaluated.  plane_cost is a function of the pixel, (n, d) and
// the hint alone, so that call would return the stored cost c (or 1e9 on an
// early abort); best_c starts at min(c, 1) <= c and only falls, so
// `c < best_c` could not hold and the result is unchanged.  In converged
// regions most propagated planes are such repeats, and they are the costly
// calls: with c near best_c they rarely abort.
// Repeat skip (with prev.flag): a neighbour whose plane the previous pass
// left unchanged offers the pixel the candidate it offered in that pass.
// Whether a candidate improves on best value b is monotone in b: at a lower b
// the abort threshold b + 0.14 and the rejection bound are lower, so a
// candidate that aborted still aborts and one that completed with cost
// C >= b still has C >= b.  In the previous pass every neighbour candidate
// was evaluated (or skipped by one of these rules), so none can improve on
// that pass's final best value; that value is the stored cost unless the
// pass refused its best plane (flag bit 1), and this pass's best value never
// exceeds the stored cost.  So with bit 1 clear, a candidate from a
// neighbour with bit 0 clear cannot win and is not evaluated.
// Register cap 72 (28 warps per SM with 64-thread blocks) measured fastest
// at 960x720 K=8: 3% ahead of 80 and 64, 10% ahead of 96.  MINB only names
// the instantiation.
template <bool COUNT, int MINB, bool PERSIST>
__global__ void __maxnreg__(72)
    pass_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start, int n_jobs, int tiles,
                unsigned int* queue, uint64_t pass, float sig_inv, float sig_n, const uint64_t* __restrict__ census,
                const float2* __restrict__ rays, PlaneBuf prev, PlaneBuf next, unsigned long long* d_work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    WorkCount wc{0, 0};
    for (int it = 0; PERSIST || it == 0; ++it) {
        const int tile = PERSIST ? next_tile(queue, tiles, it, &s_tile) : (int)blockIdx.x;
        if (tile < 0) break;
        Smem sm;
        Tile T;
        load_tile(jobs, job_start, n_jobs, tile, census, rays, smem_raw, sm, T);
        const DevJob* J = T.job;
        const int lx = threadIdx.x % T.tw, ly = threadIdx.x / T.tw;
        const int x = T.x0 + lx, y = T.y0 + ly;
        const int w = J->w, h = J->h;
        if ((int)threadIdx.x < T.tw * T.th && x < w && y < h) {
            const int nsrc = J->nsrc;
            const float total = 5.0f * 5.0f * (float)nsrc;
            const float inv_min = J->inv_min, inv_max = J->inv_max;
            const float zlo = J->zmin * 0.5f, zhi = J->zmax * 2.0f;
            const size_t base = (size_t)J->off;
            const size_t i = base + (size_t)y * w + x;
            const int stw = T.stw;
            const float2 ri = sm.ray[(ly + HALO) * stw + lx + HALO];
            uint64_t seed = pixel_rng(x, y, pass + 7);
            const float4 cur = prev.nz[i];
            const float cur_cost = prev.cost[i];
            // the offset d that cur_cost was computed with (PlaneBuf::d); a
            // propagated plane equal to (cur.n, cur_d) bit for bit would cost
            // exactly cur_cost or abort, never less, and is skipped
            const bool skip_dup = prev.d != nullptr;
            const float cur_d = skip_dup ? prev.d[i] : 0.f;
            const uint8_t* __restrict__ pflag = prev.flag;
            const bool repeat = skip_dup && pflag != nullptr && !(pflag[i] & 2);
            float best_c = cur_cost;
            float bn0 = cur.x, bn1 = cur.y, bn2 = cur.z;
            float bd = cur.w * (bn0 * ri.x + bn1 * ri.y + bn2);

            // propagation from the 4 neighbours (stereo.rs:292-321).  First
            // the gates and the duplicate test of all four, then the kept ones
            // in neighbour order: a warp runs as many plane_cost calls as its
            // busiest lane needs, not one for every neighbour some lane needs.
            // Each lane still sees its candidates, hints and best_c updates in
            // the reference's order.
            auto neighbour = [&](int q, float4& nb, float& d_plane) -> bool {
                const int ddx = q == 0 ? -1 : (q == 1 ? 1 : 0);
                const int ddy = q == 2 ? -1 : (q == 3 ? 1 : 0);
                const int xx = x + ddx, yy = y + ddy;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) return false;
                nb = prev.nz[base + (size_t)yy * w + xx];
                const float2 rj = sm.ray[(ly + HALO + ddy) * stw + lx + HALO + ddx];
                const float a_nb = nb.x * rj.x + nb.y * rj.y + nb.z;
                if (a_nb < 0.1f) return false;
                d_plane = nb.w * a_nb;
                const float a_here = nb.x * ri.x + nb.y * ri.y + nb.z;
                if (a_here < 0.1f) return false;
                const float zcand = d_plane / a_here;
                return zlo <= zcand && zcand <= zhi;
            };
            unsigned todo = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 nb;
                float d_plane;
                if (repeat) {  // an unchanged neighbour's candidate lost in the previous pass
                    const int xx = x + (q == 0 ? -1 : (q == 1 ? 1 : 0));
                    const int yy = y + (q == 2 ? -1 : (q == 3 ? 1 : 0));
                    if (xx >= 0 && yy >= 0 && xx < w && yy < h && !(pflag[base + (size_t)yy * w + xx] & 1))
                        continue;
                }
                if (!neighbour(q, nb, d_plane)) continue;
                if (skip_dup && __float_as_uint(d_plane) == __float_as_uint(cur_d) &&
                    __float_as_uint(nb.x) == __float_as_uint(cur.x) && __float_as_uint(nb.y) == __float_as_uint(cur.y) &&
                    __float_as_uint(nb.z) == __float_as_uint(cur.z))
                    continue;
                todo |= 1u << q;
            }
#pragma unroll 1
            while (todo) {
                const int q = __ffs(todo) - 1;
                todo &= todo - 1;
                float4 nb;
                float d_plane;
                neighbour(q, nb, d_plane);  // passed above; same values
                const float c = plane_cost<false, COUNT, false>(sm, stw, lx, ly, nsrc, census, nb.x, nb.y, nb.z,
                                                                      d_plane, best_c + 0.02f, total, wc, nullptr,
                                                                      skip_dup ? reject_bound(best_c, total) : INFINITY,
                                                                      skip_dup);
                if (c < best_c) {
                    best_c = c;
                    bn0 = nb.x;
                    bn1 = nb.y;
                    bn2 = nb.z;
                    bd = d_plane;
                }
            }

            // random perturbations around the current plane (stereo.rs:323-353)
    #pragma unroll 1
            for (int r = 0; r < 3; ++r) {
                const float inv = 1.0f / fmaxf(cur.w, 1e-6f);
                const float inv_new = inv + sig_inv * (inv_max - inv_min) * gauss3(seed);
                if (inv_new <= 0.0f) continue;
                const float zcand = 1.0f / inv_new;
                if (!(zlo <= zcand && zcand <= zhi)) continue;
                float nnx = cur.x + sig_n * gauss3(seed);
                float nny = cur.y + sig_n * gauss3(seed);
                float nnz = cur.z + sig_n * gauss3(seed);
                const float len = sqrtf(nnx * nnx + nny * nny + nnz * nnz);
                if (len < 1e-6f) continue;
                nnx = nnx / len;
                nny = nny / len;
                nnz = nnz / len;
                const float a_here = nnx * ri.x + nny * ri.y + nnz;
                if (a_here < 0.1f) continue;
                const float d_plane = zcand * a_here;
                const float c = plane_cost<false, COUNT, false>(sm, stw, lx, ly, nsrc, census, nnx, nny, nnz,
                                                                      d_plane, best_c + 0.02f, total, wc, nullptr,
                                                                      skip_dup ? reject_bound(best_c, total) : INFINITY,
                                                                      skip_dup);
                if (c < best_c) {
                    best_c = c;
                    bn0 = nnx;
                    bn1 = nny;
                    bn2 = nnz;
                    bd = d_plane;
                }
            }

            float4 o = cur;
            float oc = cur_cost, od = cur_d;
            uint8_t fl = 0;
            if (best_c < cur_cost) {  // stereo.rs:355-367
                const float a_here = bn0 * ri.x + bn1 * ri.y + bn2;
                if (a_here > 0.05f) {
                    o = make_float4(bn0, bn1, bn2, bd / a_here);
                    oc = fminf(best_c, 1.0f);
                    od = bd;
                    fl = 1;
                } else {
                    fl = 2;
                }
            }
            next.nz[i] = o;
            next.cost[i] = oc;
            if (skip_dup) next.d[i] = od;
            if (next.flag) next.flag[i] = fl;
        }
    }
    if (COUNT) flush_work(wc, d_work);
}

// ---------------------------------------------------------------- streamed passes
// The same pass with the tile's pixels streamed through the block's lanes.
// In pass_kernel a warp holds every candidate slot for as long as its
// slowest lane needs: most evaluations abort after a window row or two while
// a good candidate runs all 5*K rows, so most lanes wait.  Here a block of
// STREAM_THREADS threads owns a STREAM_TW x STREAM_TH tile (four pixels per
// thread) and works in two phases:
//   1. preparation, one thread per pixel: the pixel's stored plane and cost,
//      the neighbour candidates that pass the gates and the skip rules
//      (stereo.rs:292-321), and its three random perturbations drawn from
//      the pixel's RNG (stereo.rs:323-353).  The perturbations depend on the
//      stored plane alone, never on a cost, so drawing them ahead of the
//      evaluations gives the same planes.  They go to the block's slice of
//      a device scratch (48 bytes per tile pixel; the launch is persistent,
//      so a block's slice serves every tile it takes), which keeps shared
//      memory to the halo tile and lets 16 blocks share an SM.  The pass's
//      output for a pixel that accepts nothing (the carried-over plane,
//      stereo.rs:278) is written here.
//   2. evaluation: every lane advances its own candidate by one window row
//      per loop iteration; a lane whose candidate ends starts the pixel's
//      next one, and a lane whose pixel ends writes it (if a candidate beat
//      its cost) and claims the next unclaimed pixel of the tile (pixels
//      with the most candidates first; those with none are not claimed).
// Each pixel still meets its candidates, hints, rejection bounds and
// best-cost updates in the reference's order, so every output bit (and each
// work counter) is pass_kernel's.  Support-view parameters live field-major
// in shared memory (field f of view s at f * RCMVS_MAX_SOURCES + s), so lanes
// on different views read different banks and lanes on the same view read
// one broadcast word.
//
// Tile, block and register budget of the streamed passes (build-time
// settings).  Measured on the 1920x1080 K=10 workload (learned arm, depth
// maps/s): 16x16 tiles in blocks of 64 threads at 64 registers (4 pixels per
// thread, 16 blocks = 32 warps per SM) 93.9; 32x16 / 128 threads 91.3;
// 32x32 / 128 (8 pixels per thread, 7 blocks, spills) 88.6; 16x16 / 128
// (2 pixels per thread) 80.4; 32x16 / 256 76.2.  With the random candidates
// in shared memory instead of the global scratch (24 KB per block) the best
// was 16x16 / 128 at 80.0 and 16x16 / 64 reached 71.9 (9 blocks per SM).
#ifndef RCMVS_STREAM_TW
#define RCMVS_STREAM_TW 16
#define RCMVS_STREAM_TH 16
#define RCMVS_STREAM_THREADS 64
#define RCMVS_STREAM_MINB 16
#endif
constexpr int STREAM_TW = RCMVS_STREAM_TW, STREAM_TH = RCMVS_STREAM_TH;
constexpr int STREAM_PX = STREAM_TW * STREAM_TH;
constexpr int STREAM_THREADS = RCMVS_STREAM_THREADS;
static_assert(STREAM_THREADS % 32 == 0 && STREAM_TW <= 256 && STREAM_TH <= 256, "stream tile");
constexpr int STREAM_CELLS = (STREAM_TW + 2 * HALO) * (STREAM_TH + 2 * HALO);
constexpr int SF_N = 19;  // rs[9], ts[3], f, cx, cy, k, (float)w, (float)h, w (int bits)

struct StreamSmem {
    uint64_t* cen;      // halo tile
    float2* ray;        // halo tile
    const uint64_t** scp;  // [RCMVS_MAX_SOURCES] census of each support view
    float* sf;          // [SF_N][RCMVS_MAX_SOURCES]
    float* tab;         // 64 (49 used): h / 48.0f
    uint32_t* pix;      // [STREAM_PX]: lx | ly << 8 | candidate bits << 16
    float* pcost;       // [STREAM_PX] stored cost
    uint16_t* order;    // [STREAM_PX]: the claim order (pixels with candidates, most candidates first)
};

__host__ __device__ constexpr size_t stream_smem_bytes() {
    return (sizeof(uint64_t) + sizeof(float2)) * STREAM_CELLS +
           sizeof(uint64_t*) * RCMVS_MAX_SOURCES + sizeof(float) * SF_N * RCMVS_MAX_SOURCES + 64 * sizeof(float) +
           (sizeof(uint32_t) + sizeof(float) + sizeof(uint16_t)) * STREAM_PX;
}

__device__ __forceinline__ StreamSmem carve_stream(unsigned char* base) {
    StreamSmem s;
    s.cen = reinterpret_cast<uint64_t*>(base);
    s.ray = reinterpret_cast<float2*>(s.cen + STREAM_CELLS);
    s.scp = reinterpret_cast<const uint64_t**>(s.ray + STREAM_CELLS);
    s.sf = reinterpret_cast<float*>(s.scp + RCMVS_MAX_SOURCES);
    s.tab = s.sf + SF_N * RCMVS_MAX_SOURCES;
    s.pix = reinterpret_cast<uint32_t*>(s.tab + 64);
    s.pcost = reinterpret_cast<float*>(s.pix + STREAM_PX);
    s.order = reinterpret_cast<uint16_t*>(s.pcost + STREAM_PX);
    return s;
}

__device__ __forceinline__ SrcRegs load_src_fm(const StreamSmem& sm, int si) {
    const float* b = sm.sf + si;
    constexpr int S = RCMVS_MAX_SOURCES;
    SrcRegs r;
    r.rs0 = b[0 * S];
    r.rs1 = b[1 * S];
    r.rs2 = b[2 * S];
    r.rs3 = b[3 * S];
    r.rs4 = b[4 * S];
    r.rs5 = b[5 * S];
    r.rs6 = b[6 * S];
    r.rs7 = b[7 * S];
    r.rs8 = b[8 * S];
    r.ts0 = b[9 * S];
    r.ts1 = b[10 * S];
    r.ts2 = b[11 * S];
    r.f = b[12 * S];
    r.cx = b[13 * S];
    r.cy = b[14 * S];
    r.k = b[15 * S];
    r.swf = b[16 * S];
    r.shf = b[17 * S];
    r.sw = __float_as_int(b[18 * S]);
    r.sh = 0;  // not read by cost_row
    r.sc = sm.scp[si];
    return r;
}

template <bool COUNT, bool PERSIST>
#ifndef RCMVS_STREAM_MINB
#define RCMVS_STREAM_MINB (512 / RCMVS_STREAM_THREADS)
#endif
__global__ void __launch_bounds__(STREAM_THREADS, RCMVS_STREAM_MINB)
    pass_stream_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ stile_start, int n_jobs, int tiles,
                       unsigned int* queue, uint64_t pass, float sig_inv, float sig_n,
                       const uint64_t* __restrict__ census, const float2* __restrict__ rays, PlaneBuf prev,
                       PlaneBuf next, float4* __restrict__ scratch, unsigned long long* d_work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile, s_next, s_bin[8];
    const StreamSmem sm = carve_stream(smem_raw);
    // this block's slice of the random-candidate scratch: [STREAM_PX][3]
    const size_t rnd0 = (size_t)blockIdx.x * STREAM_PX * 3;
    const Smem rs{nullptr, sm.tab, sm.ray, sm.cen};  // the view cost_row reads
    constexpr int stw = STREAM_TW + 2 * HALO;
    const bool skip_dup = prev.d != nullptr;
    const uint8_t* __restrict__ pflag = prev.flag;
    const int lane = threadIdx.x & 31;
    WorkCount wc{0, 0};
    for (int it = 0; PERSIST || it == 0; ++it) {
        const int tile = PERSIST ? next_tile(queue, tiles, it, &s_tile) : (int)blockIdx.x;
        if (tile < 0) break;
        const int j = find_item(stile_start, n_jobs, tile);
        const DevJob* J = jobs + j;
        const int w = J->w, h = J->h, nsrc = J->nsrc;
        const int t = tile - stile_start[j];
        const int stx = (w + STREAM_TW - 1) / STREAM_TW;
        const int x0 = (t % stx) * STREAM_TW, y0 = (t / stx) * STREAM_TH;
        const int vw = min(STREAM_TW, w - x0), vh = min(STREAM_TH, h - y0);
        const int np = vw * vh;
        const size_t base = (size_t)J->off;

        // ---- staging: support views (field-major), h/48 table, halo tile
        for (int i = threadIdx.x; i < nsrc * SF_N; i += STREAM_THREADS) {
            const int s = i / SF_N, f = i - s * SF_N;
            const DevSrc& S = J->src[s];
            float v;
            if (f < 16)
                v = reinterpret_cast<const float*>(&S)[f];  // rs[9], ts[3], f, cx, cy, k
            else if (f == 16)
                v = (float)S.w;
            else if (f == 17)
                v = (float)S.h;
            else
                v = __int_as_float(S.w);
            sm.sf[f * RCMVS_MAX_SOURCES + s] = v;
        }
        for (int s = threadIdx.x; s < nsrc; s += STREAM_THREADS) sm.scp[s] = census + J->src[s].off;
        for (int i = threadIdx.x; i < 49; i += STREAM_THREADS) sm.tab[i] = (float)i / 48.0f;
        for (int i = threadIdx.x; i < STREAM_CELLS; i += STREAM_THREADS) {
            const int sx = i % stw, sy = i / stw;
            const int gx = min(max(x0 - HALO + sx, 0), w - 1);
            const int gy = min(max(y0 - HALO + sy, 0), h - 1);
            const size_t g = base + (size_t)gy * w + gx;
            sm.ray[i] = __ldg(rays + g);
            sm.cen[i] = __ldg(census + g);
        }
        if (threadIdx.x == 0) s_next = 0;
        if (threadIdx.x < 8) s_bin[threadIdx.x] = 0;
        __syncthreads();

        const float total = 5.0f * 5.0f * (float)nsrc;
        const float inv_min = J->inv_min, inv_max = J->inv_max;
        const float zlo = J->zmin * 0.5f, zhi = J->zmax * 2.0f;

        // ---- phase 1: prepare every pixel of the tile
        for (int p = threadIdx.x; p < np; p += STREAM_THREADS) {
            const int lx = p % vw, ly = p / vw;
            const int x = x0 + lx, y = y0 + ly;
            const size_t i = base + (size_t)y * w + x;
            const float2 ri = sm.ray[(ly + HALO) * stw + lx + HALO];
            uint64_t seed = pixel_rng(x, y, pass + 7);
            const float4 cur = prev.nz[i];
            const float cur_cost = prev.cost[i];
            const float cur_d = skip_dup ? prev.d[i] : 0.f;
            const bool repeat = skip_dup && pflag != nullptr && !(pflag[i] & 2);
            unsigned mask = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {  // the gates of pass_kernel's neighbour()
                const int ddx = q == 0 ? -1 : (q == 1 ? 1 : 0);
                const int ddy = q == 2 ? -1 : (q == 3 ? 1 : 0);
                const int xx = x + ddx, yy = y + ddy;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                const size_t ni = base + (size_t)yy * w + xx;
                if (repeat && !(pflag[ni] & 1)) continue;
                const float4 nb = prev.nz[ni];
                const float2 rj = sm.ray[(ly + HALO + ddy) * stw + lx + HALO + ddx];
                const float a_nb = nb.x * rj.x + nb.y * rj.y + nb.z;
                if (a_nb < 0.1f) continue;
                const float d_plane = nb.w * a_nb;
                const float a_here = nb.x * ri.x + nb.y * ri.y + nb.z;
                if (a_here < 0.1f) continue;
                const float zcand = d_plane / a_here;
                if (!(zlo <= zcand && zcand <= zhi)) continue;
                if (skip_dup && __float_as_uint(d_plane) == __float_as_uint(cur_d) &&
                    __float_as_uint(nb.x) == __float_as_uint(cur.x) && __float_as_uint(nb.y) == __float_as_uint(cur.y) &&
                    __float_as_uint(nb.z) == __float_as_uint(cur.z))
                    continue;
                mask |= 1u << q;
            }
#pragma unroll 1
            for (int r = 0; r < 3; ++r) {  // stereo.rs:323-353, as pass_kernel
                const float inv = 1.0f / fmaxf(cur.w, 1e-6f);
                const float inv_new = inv + sig_inv * (inv_max - inv_min) * gauss3(seed);
                if (inv_new <= 0.0f) continue;
                const float zcand = 1.0f / inv_new;
                if (!(zlo <= zcand && zcand <= zhi)) continue;
                float nnx = cur.x + sig_n * gauss3(seed);
                float nny = cur.y + sig_n * gauss3(seed);
                float nnz = cur.z + sig_n * gauss3(seed);
                const float len = sqrtf(nnx * nnx + nny * nny + nnz * nnz);
                if (len < 1e-6f) continue;
                nnx = nnx / len;
                nny = nny / len;
                nnz = nnz / len;
                const float a_here = nnx * ri.x + nny * ri.y + nnz;
                if (a_here < 0.1f) continue;
                scratch[rnd0 + p * 3 + r] = make_float4(nnx, nny, nnz, zcand * a_here);
                mask |= 16u << r;
            }
            next.nz[i] = cur;  // nothing accepted (stereo.rs:278)
            next.cost[i] = cur_cost;
            if (skip_dup) next.d[i] = cur_d;
            if (next.flag) next.flag[i] = 0;
            sm.pix[p] = (uint32_t)lx | (uint32_t)ly << 8 | mask << 16;
            sm.pcost[p] = cur_cost;
            atomicAdd(&s_bin[7 - __popc(mask)], 1);  // at most 7 candidates
        }
        __syncthreads();

        // ---- claim order: most candidates first (the longest work starts
        // early, so a tile's tail is short); pixels without candidates keep
        // the output written above and are not claimed.  Pixels are
        // independent, so the order changes no output bit.
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int b = 0; b < 8; ++b) {
                const int n = s_bin[b];
                s_bin[b] = acc;
                acc += n;
            }
        }
        __syncthreads();
        // s_bin[7] now counts the pixels with at least one candidate (read
        // at claim time: it stays fixed until the next tile's barrier)
        for (int p = threadIdx.x; p < np; p += STREAM_THREADS) {
            const int c = __popc(sm.pix[p] >> 16);
            if (c) sm.order[atomicAdd(&s_bin[7 - c], 1)] = (uint16_t)p;
        }
        __syncthreads();

        // ---- phase 2: stream the prepared pixels through the lanes
        int p = -1, cell0 = 0, si = 0, dy = 0;
        unsigned cm = 0;  // the pixel's candidates not yet started
        bool live = false, done = false;
        const size_t tb = base + (size_t)y0 * w + x0;  // the tile's first pixel
        float best_c = 0.f, bn0 = 0.f, bn1 = 0.f, bn2 = 0.f, bd = 0.f;
        float nx = 0.f, ny = 0.f, nz = 0.f, d = 0.f, sum = 0.f, thr = 0.f, rej = INFINITY;
        for (;;) {
            const bool need = !live && !done && cm == 0;
            const unsigned m = __ballot_sync(0xffffffffu, need);
            if (m) {
                if (need && p >= 0 && best_c < sm.pcost[p]) {  // stereo.rs:355-367
                    const float2 ri = sm.ray[cell0 + HALO * stw + HALO];
                    const float a_here = bn0 * ri.x + bn1 * ri.y + bn2;
                    const int lx = cell0 % stw, ly = cell0 / stw;
                    const size_t i = tb + (size_t)ly * w + lx;
                    if (a_here > 0.05f) {
                        next.nz[i] = make_float4(bn0, bn1, bn2, bd / a_here);
                        next.cost[i] = fminf(best_c, 1.0f);
                        if (skip_dup) next.d[i] = bd;
                        if (next.flag) next.flag[i] = 1;
                    } else if (next.flag) {
                        next.flag[i] = 2;
                    }
                }
                // lanes claiming together take consecutive pixels
                const int leader = __ffs(m) - 1;
                int b0 = 0;
                if (lane == leader) b0 = atomicAdd(&s_next, __popc(m));
                b0 = __shfl_sync(0xffffffffu, b0, leader);
                if (need) {
                    const int b = b0 + __popc(m & ((1u << lane) - 1u));
                    if (b >= s_bin[7]) {
                        done = true;
                    } else {
                        p = sm.order[b];
                        const uint32_t pk = sm.pix[p];
                        cell0 = (int)((pk >> 8) & 255u) * stw + (int)(pk & 255u);
                        cm = pk >> 16;
                        best_c = sm.pcost[p];
                    }
                }
            }
            if (!live && cm != 0) {  // the pixel's next candidate, in pass_kernel's order
                const int q = __ffs(cm) - 1;
                cm &= cm - 1;
                if (q < 4) {
                    const int ddx = q == 0 ? -1 : (q == 1 ? 1 : 0);
                    const int ddy = q == 2 ? -1 : (q == 3 ? 1 : 0);
                    const int lx = cell0 % stw, ly = cell0 / stw;
                    const float4 nb = prev.nz[tb + (ptrdiff_t)(ly + ddy) * w + lx + ddx];
                    const float2 rj = sm.ray[cell0 + (HALO + ddy) * stw + HALO + ddx];
                    nx = nb.x;
                    ny = nb.y;
                    nz = nb.z;
                    d = nb.w * (nb.x * rj.x + nb.y * rj.y + nb.z);
                } else {
                    const float4 c = scratch[(size_t)blockIdx.x * STREAM_PX * 3 + p * 3 + (q - 4)];
                    nx = c.x;
                    ny = c.y;
                    nz = c.z;
                    d = c.w;
                }
                sum = 0.f;
                si = 0;
                dy = 0;
                thr = (best_c + 0.02f) + 0.12f;
                rej = skip_dup ? reject_bound(best_c, total) : INFINITY;
                live = nsrc > 0;  // with no support view the cost is 0/0, never accepted
                if (COUNT) wc.evals++;
            }
            if (__all_sync(0xffffffffu, done)) break;
            if (live) {
                const SrcRegs s = load_src_fm(sm, si);
                int32_t hs = 0;
                sum = cost_row<false, false>(rs, cell0 + dy * stw, s, nx, ny, nz, d, sum, hs);
                if (COUNT) wc.rows++;
                const bool aborted = sum / abort_den(dy, si, nsrc, skip_dup) > thr || sum >= rej;
                if (aborted || (si == nsrc - 1 && dy == 4)) {
                    const float c = aborted ? 1e9f : sum / total;
                    if (c < best_c) {
                        best_c = c;
                        bn0 = nx;
                        bn1 = ny;
                        bn2 = nz;
                        bd = d;
                    }
                    live = false;
                } else if (++dy == 5) {
                    dy = 0;
                    ++si;
                }
            }
        }
    }
    if (COUNT) flush_work(wc, d_work);
}

// ---------------------------------------------------------------- split passes
// The same pass with five lanes per pixel (threads per pixel = 5, an
// autotuner axis): lane j of a pixel's group computes window column dx = j of
// every row, the group exchanges the five Hamming counts by shuffles, and
// every lane of the group adds them in dx order -- the reference's f32 chain,
// each lane holding the same sum, so the abort test and all control flow stay
// uniform within the group.  A lane keeps its column's source-independent
// values (z = d / denom and z*ray, stereo.rs:187-195) for the five rows once
// the first source has computed them, so later sources of the same candidate
// skip the divide.  Six pixels per warp (lanes 30 and 31 idle); a tile of P
// pixels runs in ceil(P / 6) warps.  Everything a pixel computes, and in
// which order, is what pass_kernel computes: the results are bit-identical.
constexpr int SPLIT = 5;     // lanes per pixel
constexpr int SPLIT_PX = 6;  // pixels per warp

template <bool COUNT>
__device__ __forceinline__ float plane_cost_split(const Smem& sm, int stw, int lx, int ly, int j, unsigned gmask,
                                                  int gbase, int nsrc, const uint64_t* __restrict__ census,
                                                  float nx, float ny, float nz, float d, float hint, float total,
                                                  WorkCount& wc, float rej, bool ahead) {
    float sum = 0.f;
    const float thr = hint + 0.12f;
    if (COUNT && j == 0) wc.evals++;
    float zc[5], xc[5], yc[5];
    unsigned dok = 0;
    for (int si = 0; si < nsrc; ++si) {
        const SrcRegs s = load_src(sm.src[si], census);
#pragma unroll
        for (int dy = 0; dy < 5; ++dy) {
            const int cell = (ly + dy) * stw + lx + j;
            if (si == 0) {
                const float2 r = sm.ray[cell];
                const float denom = nx * r.x + ny * r.y + nz;
                const float z = d / denom;
                zc[dy] = z;
                xc[dy] = z * r.x;
                yc[dy] = z * r.y;
                dok |= (denom < 0.05f ? 0u : 1u) << dy;
            }
            const float z = zc[dy], xr = xc[dy], yr = yc[dy];
            const float xs = s.rs0 * xr + s.rs1 * yr + s.rs2 * z + s.ts0;
            const float ys = s.rs3 * xr + s.rs4 * yr + s.rs5 * z + s.ts1;
            const float zs = s.rs6 * xr + s.rs7 * yr + s.rs8 * z + s.ts2;
            const float xn = xs / zs;
            const float yn = ys / zs;
            const float dist = 1.0f + s.k * (xn * xn + yn * yn);
            int u, v;
            const bool in_u = trunc_index(s.f * xn * dist + s.cx, s.swf, u);
            const bool in_v = trunc_index(s.f * yn * dist + s.cy, s.shf, v);
            const bool ok = ((dok >> dy) & 1u) && !(zs < 1e-3f) && in_u && in_v;
            const uint64_t cs = __ldg(s.sc + (ok ? (size_t)v * s.sw + u : (size_t)0));
            const int hv = __popcll(sm.cen[cell] ^ cs);
            const int h = ok ? hv : 48;
            // the row's five counts, added in dx order by every lane of the group
#pragma unroll
            for (int k = 0; k < SPLIT; ++k) sum += sm.tab[__shfl_sync(gmask, h, gbase + k)];
            if (COUNT && j == 0) wc.rows++;
            if (sum / abort_den(dy, si, nsrc, ahead) > thr || sum >= rej) return 1e9f;
        }
    }
    return sum / total;
}

// 80 registers: a few bytes spill; 96 spill nothing but leave fewer warps
// resident.
template <bool COUNT, bool PERSIST>
__global__ void __maxnreg__(80)
    pass_split_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start, int n_jobs, int tiles,
                      unsigned int* queue, uint64_t pass, float sig_inv, float sig_n,
                      const uint64_t* __restrict__ census, const float2* __restrict__ rays, PlaneBuf prev,
                      PlaneBuf next, unsigned long long* d_work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    WorkCount wc{0, 0};
    const int lane = threadIdx.x & 31;
    const int grp = lane / SPLIT, j = lane - grp * SPLIT;
    const int gbase = grp * SPLIT;
    const unsigned gmask = 0x1Fu << gbase;
    const int p = (int)(threadIdx.x >> 5) * SPLIT_PX + grp;  // the group's pixel in the tile
    for (int it = 0; PERSIST || it == 0; ++it) {
        const int tile = PERSIST ? next_tile(queue, tiles, it, &s_tile) : (int)blockIdx.x;
        if (tile < 0) break;
        Smem sm;
        Tile T;
        load_tile(jobs, job_start, n_jobs, tile, census, rays, smem_raw, sm, T);
        const DevJob* J = T.job;
        const int lx = p % T.tw, ly = p / T.tw;
        const int x = T.x0 + lx, y = T.y0 + ly;
        const int w = J->w, h = J->h;
        if (lane < SPLIT * SPLIT_PX && p < T.tw * T.th && x < w && y < h) {
            const int nsrc = J->nsrc;
            const float total = 5.0f * 5.0f * (float)nsrc;
            const float inv_min = J->inv_min, inv_max = J->inv_max;
            const float zlo = J->zmin * 0.5f, zhi = J->zmax * 2.0f;
            const size_t base = (size_t)J->off;
            const size_t i = base + (size_t)y * w + x;
            const int stw = T.stw;
            const float2 ri = sm.ray[(ly + HALO) * stw + lx + HALO];
            uint64_t seed = pixel_rng(x, y, pass + 7);
            const float4 cur = prev.nz[i];
            const float cur_cost = prev.cost[i];
            const bool skip_dup = prev.d != nullptr;
            const float cur_d = skip_dup ? prev.d[i] : 0.f;
            const uint8_t* __restrict__ pflag = prev.flag;
            const bool repeat = skip_dup && pflag != nullptr && !(pflag[i] & 2);
            float best_c = cur_cost;
            float bn0 = cur.x, bn1 = cur.y, bn2 = cur.z;
            float bd = cur.w * (bn0 * ri.x + bn1 * ri.y + bn2);
            auto neighbour = [&](int q, float4& nb, float& d_plane) -> bool {
                const int ddx = q == 0 ? -1 : (q == 1 ? 1 : 0);
                const int ddy = q == 2 ? -1 : (q == 3 ? 1 : 0);
                const int xx = x + ddx, yy = y + ddy;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) return false;
                nb = prev.nz[base + (size_t)yy * w + xx];
                const float2 rj = sm.ray[(ly + HALO + ddy) * stw + lx + HALO + ddx];
                const float a_nb = nb.x * rj.x + nb.y * rj.y + nb.z;
                if (a_nb < 0.1f) return false;
                d_plane = nb.w * a_nb;
                const float a_here = nb.x * ri.x + nb.y * ri.y + nb.z;
                if (a_here < 0.1f) return false;
                const float zcand = d_plane / a_here;
                return zlo <= zcand && zcand <= zhi;
            };
            unsigned todo = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 nb;
                float d_plane;
                if (repeat) {  // an unchanged neighbour's candidate lost in the previous pass
                    const int xx = x + (q == 0 ? -1 : (q == 1 ? 1 : 0));
                    const int yy = y + (q == 2 ? -1 : (q == 3 ? 1 : 0));
                    if (xx >= 0 && yy >= 0 && xx < w && yy < h && !(pflag[base + (size_t)yy * w + xx] & 1))
                        continue;
                }
                if (!neighbour(q, nb, d_plane)) continue;
                if (skip_dup && __float_as_uint(d_plane) == __float_as_uint(cur_d) &&
                    __float_as_uint(nb.x) == __float_as_uint(cur.x) && __float_as_uint(nb.y) == __float_as_uint(cur.y) &&
                    __float_as_uint(nb.z) == __float_as_uint(cur.z))
                    continue;
                todo |= 1u << q;
            }
#pragma unroll 1
            while (todo) {
                const int q = __ffs(todo) - 1;
                todo &= todo - 1;
                float4 nb;
                float d_plane;
                neighbour(q, nb, d_plane);
                const float c = plane_cost_split<COUNT>(sm, stw, lx, ly, j, gmask, gbase, nsrc, census, nb.x, nb.y,
                                                        nb.z, d_plane, best_c + 0.02f, total, wc,
                                                        skip_dup ? reject_bound(best_c, total) : INFINITY, skip_dup);
                if (c < best_c) {
                    best_c = c;
                    bn0 = nb.x;
                    bn1 = nb.y;
                    bn2 = nb.z;
                    bd = d_plane;
                }
            }
#pragma unroll 1
            for (int r = 0; r < 3; ++r) {
                const float inv = 1.0f / fmaxf(cur.w, 1e-6f);
                const float inv_new = inv + sig_inv * (inv_max - inv_min) * gauss3(seed);
                if (inv_new <= 0.0f) continue;
                const float zcand = 1.0f / inv_new;
                if (!(zlo <= zcand && zcand <= zhi)) continue;
                float nnx = cur.x + sig_n * gauss3(seed);
                float nny = cur.y + sig_n * gauss3(seed);
                float nnz = cur.z + sig_n * gauss3(seed);
                const float len = sqrtf(nnx * nnx + nny * nny + nnz * nnz);
                if (len < 1e-6f) continue;
                nnx = nnx / len;
                nny = nny / len;
                nnz = nnz / len;
                const float a_here = nnx * ri.x + nny * ri.y + nnz;
                if (a_here < 0.1f) continue;
                const float d_plane = zcand * a_here;
                const float c = plane_cost_split<COUNT>(sm, stw, lx, ly, j, gmask, gbase, nsrc, census, nnx, nny,
                                                        nnz, d_plane, best_c + 0.02f, total, wc,
                                                        skip_dup ? reject_bound(best_c, total) : INFINITY, skip_dup);
                if (c < best_c) {
                    best_c = c;
                    bn0 = nnx;
                    bn1 = nny;
                    bn2 = nnz;
                    bd = d_plane;
                }
            }
            if (j == 0) {
                float4 o = cur;
                float oc = cur_cost, od = cur_d;
                uint8_t fl = 0;
                if (best_c < cur_cost) {  // stereo.rs:355-367
                    const float a_here = bn0 * ri.x + bn1 * ri.y + bn2;
                    if (a_here > 0.05f) {
                        o = make_float4(bn0, bn1, bn2, bd / a_here);
                        oc = fminf(best_c, 1.0f);
                        od = bd;
                        fl = 1;
                    } else {
                        fl = 2;
                    }
                }
                next.nz[i] = o;
                next.cost[i] = oc;
                if (skip_dup) next.d[i] = od;
                if (next.flag) next.flag[i] = fl;
            }
        }
    }
    if (COUNT) flush_work(wc, d_work);
}

// ---------------------------------------------------------------- row-step kernels
// The same init and pass computations with per-thread candidate streams
// advanced one 5-term window row per loop iteration: a lane whose candidate
// aborts early starts its next candidate at once instead of idling until
// every lane of the warp has finished the current one.  Each candidate's
// rows, abort tests, hint and best-cost bookkeeping happen in the
// reference's order, so results are bit-identical to the kernels above.

__device__ __forceinline__ float hyp_depth(float inv_min, float inv_max, int hi, int nh) {
    const float inv = inv_min + (inv_max - inv_min) * (float)hi / (float)(nh - 1);  // stereo.rs:259-260
    return 1.0f / inv;
}

template <bool COUNT, int MINB, bool PERSIST>
__global__ void __launch_bounds__(256, MINB)
    init_rows_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start, int n_jobs, int tiles,
                     unsigned int* queue, int nh, const uint64_t* __restrict__ census, const float2* __restrict__ rays,
                     PlaneBuf out, unsigned long long* d_work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    WorkCount wc{0, 0};
    for (int it = 0; PERSIST || it == 0; ++it) {
        const int tile = PERSIST ? next_tile(queue, tiles, it, &s_tile) : (int)blockIdx.x;
        if (tile < 0) break;
        Smem sm;
        Tile T;
        load_tile(jobs, job_start, n_jobs, tile, census, rays, smem_raw, sm, T);
        const DevJob* J = T.job;
        const int lx = threadIdx.x % T.tw, ly = threadIdx.x / T.tw;
        const int x = T.x0 + lx, y = T.y0 + ly;
        const bool inside = (int)threadIdx.x < T.tw * T.th && x < J->w && y < J->h;
        const int nsrc = J->nsrc;
        const float total = 5.0f * 5.0f * (float)nsrc;
        const float inv_min = J->inv_min, inv_max = J->inv_max;
        float best_c = INFINITY, best_d = 0.f;
        int hi = 0, si = 0, dy = 0;
        float d = hyp_depth(inv_min, inv_max, 0, nh);
        float sum = 0.f;
        float thr = INFINITY;  // (best_c + 0.02) + 0.12 with best_c = +inf
        float rej = INFINITY;  // early-rejection bound (reject_bound)
        const bool early = out.d != nullptr;  // off for the reference call sequence
        int32_t hs = 0;
        bool live = inside;
        if (COUNT && live) wc.evals++;
        while (live) {
            bool fin = true, aborted = false;
            if (nsrc > 0) {
                const SrcRegs s = load_src(sm.src[si], census);
                sum = cost_row<true, false>(sm, (ly + dy) * T.stw + lx, s, 0.f, 0.f, 1.f, d, sum, hs);
                if (COUNT) wc.rows++;
                aborted = sum / abort_den(dy, si, nsrc, early) > thr || sum >= rej;
                fin = aborted || (si == nsrc - 1 && dy == 4);
            }
            if (fin) {
                const float c = aborted ? 1e9f : sum / total;
                if (c < best_c) {
                    best_c = c;
                    best_d = d;
                }
                if (++hi >= nh) {
                    live = false;
                } else {
                    d = hyp_depth(inv_min, inv_max, hi, nh);
                    sum = 0.f;
                    si = 0;
                    dy = 0;
                    thr = (best_c + 0.02f) + 0.12f;
                    if (early) rej = reject_bound(best_c, total);
                    if (COUNT) wc.evals++;
                }
            } else if (++dy == 5) {
                dy = 0;
                ++si;
            }
        }
        if (inside) {
            const size_t i = (size_t)J->off + (size_t)y * J->w + x;
            out.nz[i] = make_float4(0.0f, 0.0f, 1.0f, best_d);
            out.cost[i] = fminf(best_c, 1.0f);
            if (out.d) out.d[i] = best_d;  // n = (0,0,1): d = z
        }
    }
    if (COUNT) flush_work(wc, d_work);
}

// ---------------------------------------------------------------- table init
// The plane sweep with the window counts shared between pixels.  On a
// fronto-parallel plane (n = (0,0,1), so denom = 1 and z = d for every
// window cell) the count of a window cell -- where its ray at depth d lands
// in a source and the Hamming distance to the census there -- depends on the
// cell, the hypothesis and the source only, not on which pixel's window
// holds it.  So the block walks the hypotheses together: for hypothesis hi
// and source si it computes the count of every cell of the tile and its
// halo once into shared memory (a tile of 64 pixels has 144 cells instead
// of 64 x 25 window terms), then every pixel runs the reference's serial f32
// chain for that source -- its five counts per row added in dx order, the
// abort test and the early rejection after each row -- reading the counts
// from the table.  A source's table is built only while some pixel of the
// block still needs it, so hypotheses that every pixel drops early cost
// little.  Each pixel's chain, hints and best-cost updates are those of
// stereo.rs:247-269: the results are bit-identical to init_rows_kernel.
constexpr int TABLE_CELLS = 1312;  // (tw + 4) x (th + 4) for every tile shape of at most 256 pixels

template <bool COUNT, bool PERSIST>
__global__ void __launch_bounds__(256)
    init_table_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start, int n_jobs,
                      int tiles, unsigned int* queue, int nh, const uint64_t* __restrict__ census,
                      const float2* __restrict__ rays, PlaneBuf out, unsigned long long* d_work) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    __shared__ uint8_t s_h[TABLE_CELLS];
    WorkCount wc{0, 0};
    for (int it = 0; PERSIST || it == 0; ++it) {
        const int tile = PERSIST ? next_tile(queue, tiles, it, &s_tile) : (int)blockIdx.x;
        if (tile < 0) break;
        Smem sm;
        Tile T;
        load_tile(jobs, job_start, n_jobs, tile, census, rays, smem_raw, sm, T);
        const DevJob* J = T.job;
        const int lx = threadIdx.x % T.tw, ly = threadIdx.x / T.tw;
        const int x = T.x0 + lx, y = T.y0 + ly;
        const bool inside = (int)threadIdx.x < T.tw * T.th && x < J->w && y < J->h;
        const int nsrc = J->nsrc;
        const float total = 5.0f * 5.0f * (float)nsrc;
        const float inv_min = J->inv_min, inv_max = J->inv_max;
        const bool early = out.d != nullptr;  // off for the reference call sequence
        const int cells = T.stw * (T.th + 2 * HALO);
        float best_c = INFINITY, best_d = 0.f;
        for (int hi = 0; hi < nh; ++hi) {
            const float d = hyp_depth(inv_min, inv_max, hi, nh);
            const float thr = (best_c + 0.02f) + 0.12f;  // +inf before the first hypothesis
            const float rej = early ? reject_bound(best_c, total) : INFINITY;
            bool alive = inside;
            float sum = 0.f;
            if (COUNT && inside) wc.evals++;
            for (int si = 0; si < nsrc; ++si) {
                if (!__syncthreads_or(alive)) break;  // also: the previous table is no longer read
                const SrcRegs s = load_src(sm.src[si], census);
                for (int c = threadIdx.x; c < cells; c += blockDim.x) {
                    const float2 r = sm.ray[c];
                    const float xr = d * r.x;
                    const float yr = d * r.y;
                    const float xs = s.rs0 * xr + s.rs1 * yr + s.rs2 * d + s.ts0;
                    const float ys = s.rs3 * xr + s.rs4 * yr + s.rs5 * d + s.ts1;
                    const float zs = s.rs6 * xr + s.rs7 * yr + s.rs8 * d + s.ts2;
                    const float xn = xs / zs;
                    const float yn = ys / zs;
                    const float dist = 1.0f + s.k * (xn * xn + yn * yn);
                    int u, v;
                    const bool in_u = trunc_index(s.f * xn * dist + s.cx, s.swf, u);
                    const bool in_v = trunc_index(s.f * yn * dist + s.cy, s.shf, v);
                    const bool ok = !(zs < 1e-3f) && in_u && in_v;  // denom = 1 >= 0.05
                    const uint64_t cs = __ldg(s.sc + (ok ? (size_t)v * s.sw + u : (size_t)0));
                    s_h[c] = ok ? (uint8_t)__popcll(sm.cen[c] ^ cs) : (uint8_t)48;
                }
                __syncthreads();
                if (alive) {
            #pragma unroll
                    for (int dy = 0; dy < 5; ++dy) {
                        const int row = (ly + dy) * T.stw + lx;
#pragma unroll
                        for (int dx = 0; dx < 5; ++dx) sum += sm.tab[s_h[row + dx]];
                        if (COUNT) wc.rows++;
                        if (sum / abort_den(dy, si, nsrc, early) > thr || sum >= rej) {
                            alive = false;
                            break;
                        }
                    }
                }
            }
            if (inside) {
                const float c = alive ? sum / total : 1e9f;
                if (c < best_c) {
                    best_c = c;
                    best_d = d;
                }
            }
        }
        if (inside) {
            const size_t i = (size_t)J->off + (size_t)y * J->w + x;
            out.nz[i] = make_float4(0.0f, 0.0f, 1.0f, best_d);
            out.cost[i] = fminf(best_c, 1.0f);
            if (out.d) out.d[i] = best_d;  // n = (0,0,1): d = z
        }
    }
    if (COUNT) flush_work(wc, d_work);
}

// ---------------------------------------------------------------- learned init
// Patch-match init from learned proposals (no reference counterpart).  A
// pixel whose quarter-resolution cell predicts a plane with confidence
// sigmoid(logit) >= conf_thr (tested as logit >= logit_thr, the threshold's
// logit, computed once on the host) tries n_local planes with the predicted normal
// and inverse depths evenly spread over +-span/2 (in fractions of
// [1/zmax, 1/zmin]) around the prediction, each kept only if it passes the
// reference's gates (positive inverse depth, depth in [zmin/2, 2 zmax],
// n . ray >= 0.1), scored by plane_cost with the sweep's early-abort hint;
// the best one seeds the pixel.  A predicted depth is placed on the ray of
// the cell's anchor pixel, so all pixels of a cell start from the same
// plane (n, d): propagation between them then repeats planes that the pass
// skips (C5: passes 1.83 -> 1.57 s per step, GT accuracy unchanged to 5
// digits; per-pixel depths gave the same accuracy).  Every other pixel (and a confident one whose
// local planes all fail the gates) runs the 64-plane sweep of
// stereo.rs:247-269 unchanged.
// Two phases per tile.  First each confident lane streams its local planes
// one window row per step.  Then the tile's remaining pixels are listed in
// shared memory and the block's threads take them in turn for the sweep
// (fronto-parallel, as init_rows_kernel): a few low-confidence pixels
// scattered over a tile occupy one warp's lanes together instead of holding
// every warp that contains one for all 64 hypotheses.  Every pixel's
// computation is the same; only which thread does it changes.
// Phase 1's table (init_learned_rows_kernel).  The quarter cells that meet a
// tile of at most 256 pixels number at most 64 (a 256 x 1 or 1 x 256 tile;
// tiles start at multiples of their sides), and the window boxes of their
// pixels hold at most (tw + 4 x cell columns) x (th + 4 x cell rows) cells,
// 2560 for those two shapes, the largest.
constexpr int LT_SLOTS = 72;
constexpr int LT_ENTRIES = 2624;

// 64 registers (4 blocks of 256 threads; with the default 8x8 tiles, 16
// blocks = 32 warps per SM): on the 1920x1080 K=10 workload 164 -> 152 ms
// per step against 80 registers, whose 24 resident warps per SM left this
// latency-bound kernel short of warps; the few extra spills cost less.
template <bool PERSIST>
__global__ void __launch_bounds__(256, 4)
    init_learned_rows_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start, int n_jobs,
                             int tiles, unsigned int* queue, int nh, const uint64_t* __restrict__ census,
                             const float2* __restrict__ rays, PlaneBuf out, const float* __restrict__ pred,
                             const int64_t* __restrict__ pred_off, float logit_thr, int n_local, float span,
                             int sweep_seeded, unsigned long long* d_learned) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    __shared__ int s_n;
    __shared__ unsigned short s_list[256];
    __shared__ float s_seed_cost[256];  // phase 1's best cost per tile pixel (+inf: not seeded)
    // phase 1's table: per quarter cell of the tile (slot), the box of window
    // cells its seeded pixels read, the cell's current plane, and the counts
    __shared__ int s_bx0[LT_SLOTS], s_bx1[LT_SLOTS], s_by0[LT_SLOTS], s_by1[LT_SLOTS];
    __shared__ int s_off[LT_SLOTS + 1];
    __shared__ int s_epoch[LT_SLOTS];
    __shared__ float4 s_pl[LT_SLOTS];
    __shared__ uint8_t s_cnt[LT_ENTRIES];
    for (int it = 0; PERSIST || it == 0; ++it) {
        const int tile = PERSIST ? next_tile(queue, tiles, it, &s_tile) : (int)blockIdx.x;
        if (tile < 0) break;
        Smem sm;
        Tile T;
        load_tile(jobs, job_start, n_jobs, tile, census, rays, smem_raw, sm, T);
        if (threadIdx.x == 0) s_n = 0;
        const DevJob* J = T.job;
        const int j = (int)(J - jobs);
        const int lx = threadIdx.x % T.tw, ly = threadIdx.x / T.tw;
        const int x = T.x0 + lx, y = T.y0 + ly;
        const bool inside = (int)threadIdx.x < T.tw * T.th && x < J->w && y < J->h;
        const int nsrc = J->nsrc;
        const float total = 5.0f * 5.0f * (float)nsrc;
        const float zlo = J->zmin * 0.5f, zhi = J->zmax * 2.0f;
        const float inv_min = J->inv_min, inv_max = J->inv_max, span_inv = inv_max - inv_min;
        const float2 ri = inside ? sm.ray[(ly + HALO) * T.stw + lx + HALO] : make_float2(0.f, 0.f);
        // this lane's prediction
        bool learned = false;
        float pnx = 0.f, pny = 0.f, pnz = 1.f, pa = 1.f, pac = 1.f, t0 = 0.f;
        const int wq = J->w >> 2, hq = J->h >> 2;
        int qx = 0, qy = 0;
        if (inside && wq > 0 && hq > 0) {
            qx = min(x >> 2, wq - 1);
            qy = min(y >> 2, hq - 1);
            const float* o = pred + (pred_off[j] + (int64_t)qy * wq + qx) * NET_OUT_C;
            const float len = sqrtf(o[1] * o[1] + o[2] * o[2] + o[3] * o[3]);
            if (o[4] >= logit_thr && len > 1e-6f) {
                pnx = o[1] / len;
                pny = o[2] / len;
                pnz = o[3] / len;
                pa = pnx * ri.x + pny * ri.y + pnz;
                t0 = o[0];
                learned = pa >= 0.1f;
                // the cell's anchor pixel (4qx+1, 4qy+1): the predicted depth
                // is placed on its ray, so every pixel of the cell gets the
                // same plane (n, d)
                const float2 rc = __ldg(rays + (size_t)J->off + (size_t)(4 * qy + 1) * J->w + 4 * qx + 1);
                pac = pnx * rc.x + pny * rc.y + pnz;
                learned = learned && pac >= 0.1f;
            }
        }

        // phase 1: the local planes of the confident pixels.  Every pixel of
        // a quarter cell that is seeded evaluates the cell's plane (n, d), so
        // a window cell's count under it -- where the cell's ray meets the
        // plane, where that point lands in a source, the Hamming distance
        // there -- is the same for every pixel whose window holds the cell.
        // Per local plane and source the block computes, for each quarter
        // cell of the tile (a slot), the counts of the box of window cells
        // its seeded pixels read, once, into shared memory; then each pixel
        // runs the reference's chain (five counts per row in dx order, the
        // abort test, the early rejection) over them.  A source's counts are
        // computed only for slots that still have a pixel evaluating.
        const int qx0 = wq > 0 ? min(T.x0 >> 2, wq - 1) : 0, qy0 = hq > 0 ? min(T.y0 >> 2, hq - 1) : 0;
        const int qx1 = wq > 0 ? min((min(T.x0 + T.tw, J->w) - 1) >> 2, wq - 1) : 0;
        const int ncx = qx1 - qx0 + 1;
        const int slot = learned ? (qy - qy0) * ncx + (qx - qx0) : -1;
        for (int q = threadIdx.x; q < LT_SLOTS; q += blockDim.x) {
            s_bx0[q] = INT_MAX;
            s_bx1[q] = INT_MIN;
            s_by0[q] = INT_MAX;
            s_by1[q] = INT_MIN;
            s_epoch[q] = 0;
        }
        __syncthreads();  // also: s_n = 0 is visible
        if (learned) {  // the window cells of this pixel, in shared-tile coordinates
            atomicMin(&s_bx0[slot], lx);
            atomicMax(&s_bx1[slot], lx + 2 * HALO);
            atomicMin(&s_by0[slot], ly);
            atomicMax(&s_by1[slot], ly + 2 * HALO);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int o = 0;
            for (int q = 0; q < LT_SLOTS; ++q) {
                s_off[q] = o;
                if (s_bx1[q] >= s_bx0[q]) o += (s_bx1[q] - s_bx0[q] + 1) * (s_by1[q] - s_by0[q] + 1);
            }
            s_off[LT_SLOTS] = o;
        }
        __syncthreads();
        const int n_entries = s_off[LT_SLOTS];
        bool any_local = false;
        float best_c = INFINITY;
        float4 plane = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
        float plane_d = 0.f;
        const bool early = out.d != nullptr;  // early rejection off for the reference call sequence
        int32_t hs = 0;
        for (int k = 0; k < n_local; ++k) {
            // this pixel's plane k: the cell's predicted depth on the anchor
            // ray, the cell's offset d, this pixel's depth
            bool ev = false;
            float zi = 0.f, dcell = 0.f;
            if (learned) {
                const float tk = t0 + span * ((float)k / (float)max(n_local - 1, 1) - 0.5f);
                const float inv = inv_min + tk * span_inv;
                if (inv > 0.f) {
                    const float z = 1.f / inv;  // depth on the anchor ray
                    dcell = z * pac;
                    zi = dcell / pa;  // depth on this pixel's ray
                    ev = zi >= zlo && zi <= zhi;
                    s_pl[slot] = make_float4(pnx, pny, pnz, dcell);  // the same values from every pixel of the cell
                }
            }
            any_local = any_local || ev;
            const float thr = (best_c + 0.02f) + 0.12f;  // +inf for the first plane
            const float rej = early ? reject_bound(best_c, total) : INFINITY;
            bool alive = ev;
            float sum = 0.f;
            for (int si = 0; si < nsrc; ++si) {
                const int epoch = k * 64 + si + 1;
                if (alive) s_epoch[slot] = epoch;
                if (!__syncthreads_or(alive)) break;  // also: the previous counts are no longer read
                const SrcRegs s = load_src(sm.src[si], census);
                for (int e = threadIdx.x; e < n_entries; e += blockDim.x) {
                    int q = 0;
                    while (s_off[q + 1] <= e) ++q;  // the slot of entry e
                    if (s_epoch[q] != epoch) continue;
                    const int bw = s_bx1[q] - s_bx0[q] + 1;
                    const int r = e - s_off[q];
                    const int c = (s_by0[q] + r / bw) * T.stw + s_bx0[q] + r % bw;
                    const float4 pl = s_pl[q];
                    // one window term of cost_row (stereo.rs:185-213)
                    const float2 rr = sm.ray[c];
                    const float denom = pl.x * rr.x + pl.y * rr.y + pl.z;
                    const float z = pl.w / denom;
                    const float xr = z * rr.x;
                    const float yr = z * rr.y;
                    const float xs = s.rs0 * xr + s.rs1 * yr + s.rs2 * z + s.ts0;
                    const float ys = s.rs3 * xr + s.rs4 * yr + s.rs5 * z + s.ts1;
                    const float zs = s.rs6 * xr + s.rs7 * yr + s.rs8 * z + s.ts2;
                    const float xn = xs / zs;
                    const float yn = ys / zs;
                    const float dist = 1.0f + s.k * (xn * xn + yn * yn);
                    int u, v;
                    const bool in_u = trunc_index(s.f * xn * dist + s.cx, s.swf, u);
                    const bool in_v = trunc_index(s.f * yn * dist + s.cy, s.shf, v);
                    const bool ok = !(denom < 0.05f) && !(zs < 1e-3f) && in_u && in_v;
                    const uint64_t cs = __ldg(s.sc + (ok ? (size_t)v * s.sw + u : (size_t)0));
                    s_cnt[e] = ok ? (uint8_t)__popcll(sm.cen[c] ^ cs) : (uint8_t)48;
                }
                __syncthreads();
                if (alive) {
                                const int bw = s_bx1[slot] - s_bx0[slot] + 1;
                    const int base = s_off[slot] + (ly - s_by0[slot]) * bw + (lx - s_bx0[slot]);
#pragma unroll
                    for (int dy = 0; dy < 5; ++dy) {
#pragma unroll
                        for (int dx = 0; dx < 5; ++dx) sum += sm.tab[s_cnt[base + dy * bw + dx]];
                        if (sum / abort_den(dy, si, nsrc, early) > thr || sum >= rej) {
                            alive = false;
                            break;
                        }
                    }
                }
            }
            if (ev) {
                const float c = alive ? sum / total : 1e9f;
                if (c < best_c) {
                    best_c = c;
                    plane = make_float4(pnx, pny, pnz, zi);
                    plane_d = dcell;
                }
            }
        }
        (void)hs;
        const bool seeded = inside && learned && any_local;
        if (seeded) {
            const size_t i = (size_t)J->off + (size_t)y * J->w + x;
            out.nz[i] = plane;
            out.cost[i] = fminf(best_c, 1.0f);
            if (out.d) out.d[i] = plane_d;
        }
        if ((int)threadIdx.x < 256) s_seed_cost[threadIdx.x] = seeded ? best_c : INFINITY;
        if (inside && (!seeded || sweep_seeded)) s_list[atomicAdd(&s_n, 1)] = (unsigned short)threadIdx.x;
        const unsigned bal = __ballot_sync(0xffffffffu, seeded);
        if ((threadIdx.x & 31) == 0 && bal) atomicAdd(d_learned, (unsigned long long)__popc(bal));
        __syncthreads();  // the list is complete

        // phase 2: the plane sweep (stereo.rs:247-269) of the listed pixels
        const int n_list = s_n;
        for (int e = threadIdx.x; e < n_list; e += blockDim.x) {
            const int pt = s_list[e];
            const int plx = pt % T.tw, ply = pt / T.tw;
            const int px = T.x0 + plx, py = T.y0 + ply;
            // a seeded pixel (sweep_seeded) starts the sweep from its
            // proposal's cost: the sweep's hint rule then holds from the first
            // hypothesis, and a sweep plane replaces the proposal only when
            // strictly cheaper
            float bc = s_seed_cost[pt], bdep = 0.f;
            bool improved = false;
            int hi = 0, ssi = 0, sdy = 0;
            float d = hyp_depth(inv_min, inv_max, 0, nh);
            float ssum = 0.f, sthr = (bc + 0.02f) + 0.12f;
            float srej = early ? reject_bound(bc, total) : INFINITY;
            bool slive = true;
            while (slive) {
                bool fin = true, aborted = false;
                if (nsrc > 0) {
                    const SrcRegs s = load_src(sm.src[ssi], census);
                    ssum = cost_row<true, false>(sm, (ply + sdy) * T.stw + plx, s, 0.f, 0.f, 1.f, d, ssum, hs);
                    aborted = ssum / abort_den(sdy, ssi, nsrc, early) > sthr || ssum >= srej;
                    fin = aborted || (ssi == nsrc - 1 && sdy == 4);
                }
                if (fin) {
                    const float c = aborted ? 1e9f : ssum / total;
                    if (c < bc) {
                        bc = c;
                        bdep = d;
                        improved = true;
                    }
                    if (++hi >= nh) {
                        slive = false;
                    } else {
                        d = hyp_depth(inv_min, inv_max, hi, nh);
                        ssum = 0.f;
                        ssi = 0;
                        sdy = 0;
                        sthr = (bc + 0.02f) + 0.12f;
                        if (early) srej = reject_bound(bc, total);
                    }
                } else if (++sdy == 5) {
                    sdy = 0;
                    ++ssi;
                }
            }
            if (improved || !(s_seed_cost[pt] < INFINITY)) {
                const size_t i = (size_t)J->off + (size_t)py * J->w + px;
                out.nz[i] = make_float4(0.0f, 0.0f, 1.0f, bdep);
                out.cost[i] = fminf(bc, 1.0f);
                if (out.d) out.d[i] = bdep;
            }
        }
    }
}

// ---------------------------------------------------------------- gate
// stereo.rs:373-393 (+ normals, an extension)
__global__ void gate_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start, int n_jobs,
                            float cost_thr, const uint64_t* __restrict__ census, PlaneBuf planes,
                            float* __restrict__ depth, float* __restrict__ cost, float* __restrict__ normal) {
    const int j = find_item(job_start, n_jobs, blockIdx.x);
    const DevJob* J = jobs + j;
    const int tw = J->tw, th = J->th;
    if ((int)threadIdx.x >= tw * th) return;
    const int t = blockIdx.x - job_start[j];
    const int x = (t % J->tiles_x) * tw + (int)threadIdx.x % tw;
    const int y = (t / J->tiles_x) * th + (int)threadIdx.x / tw;
    if (x >= J->w || y >= J->h) return;
    const size_t i = (size_t)J->off + (size_t)y * J->w + x;
    const float4 p = planes.nz[i];
    const float c = planes.cost[i];
    const int tex = __popcll(census[i]);
    const bool textured = tex >= 4 && tex <= 44;
    const bool ok = textured && c < cost_thr && p.w > J->zmin * 0.5f && p.w < J->zmax * 2.0f;
    depth[i] = ok ? p.w : 0.0f;
    cost[i] = c;
    if (normal) {
        normal[3 * i] = p.x;
        normal[3 * i + 1] = p.y;
        normal[3 * i + 2] = p.z;
    }
}

// ---------------------------------------------------------------- diagnostics
__global__ void cost_field_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ job_start,
                                  const uint64_t* __restrict__ census, const float2* __restrict__ rays,
                                  const float4* __restrict__ planes, const float* __restrict__ hints,
                                  float* __restrict__ cost_out, int32_t* __restrict__ hsum_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem sm;
    Tile T;
    load_tile(jobs, job_start, 1, blockIdx.x, census, rays, smem_raw, sm, T);
    const DevJob* J = T.job;
    const int lx = threadIdx.x % T.tw, ly = threadIdx.x / T.tw;
    const int x = T.x0 + lx, y = T.y0 + ly;
    if ((int)threadIdx.x >= T.tw * T.th || x >= J->w || y >= J->h) return;
    const size_t li = (size_t)y * J->w + x;
    const float4 p = planes[li];
    WorkCount wc{0, 0};
    int32_t hs = 0;
    const float total = 5.0f * 5.0f * (float)J->nsrc;
    cost_out[li] = plane_cost<false, false, true>(sm, T.stw, lx, ly, J->nsrc, census, p.x, p.y, p.z, p.w,
                                                  hints[li], total, wc, &hs);
    hsum_out[li] = hs;
}

__global__ void f2i_kernel(const float* in, int n, int32_t* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2int_rz(in[i]);
}

}  // namespace

size_t stereo_smem_bytes(TileShape ts) { return smem_bytes(ts.tw, ts.th); }

// Threads of a split-pass block for tiles of up to `px` pixels.
int split_threads(int px) { return 32 * ((px + SPLIT_PX - 1) / SPLIT_PX); }

int stream_tiles(int w, int h) { return ((w + STREAM_TW - 1) / STREAM_TW) * ((h + STREAM_TH - 1) / STREAM_TH); }

LaunchGeom stream_geom(int tiles) {
    LaunchGeom g{STREAM_THREADS, stream_smem_bytes(), tiles, nullptr};
    g.stream = true;
    return g;
}


size_t stream_scratch_bytes(int blocks) { return sizeof(float4) * STREAM_PX * 3 * (size_t)blocks; }

namespace {
// Blocks of a persistent launch: as many as stay resident on all SMs at
// once (the queue hands out the tiles), never more than there are tiles.
template <typename K>
int launch_grid(K kernel, const LaunchGeom& g) {
    if (!g.queue) return g.tiles;
    int dev = 0, nsm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, g.nthr, g.smem) != cudaSuccess) {
        (void)cudaGetLastError();
        return g.tiles;  // any grid size is correct with a queue
    }
    const long long n = (long long)std::max(per_sm, 1) * std::max(nsm, 1);
    return (int)std::min<long long>(n, g.tiles);
}
}  // namespace

int stereo_resident_grid(const LaunchGeom& g) { return launch_grid(pass_kernel<false, 3, true>, g); }
int stream_grid(const LaunchGeom& g) {
    LaunchGeom q = g;
    unsigned int dummy = 0;
    q.queue = &dummy;  // any non-null queue: the resident grid
    return std::max(launch_grid(pass_stream_kernel<false, true>, q), 1);
}

namespace {
template <bool COUNT, bool PERSIST>
void init_as(int variant, const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g, int nh,
             const uint64_t* census, const float2* rays, PlaneBuf out, unsigned long long* d_work, cudaStream_t st) {
    if (variant == 1)
        init_kernel<COUNT, PERSIST><<<launch_grid(init_kernel<COUNT, PERSIST>, g), g.nthr, g.smem, st>>>(
            d_jobs, d_job_start, n_jobs, g.tiles, g.queue, nh, census, rays, out, d_work);
    else if (variant == 2)
        init_table_kernel<COUNT, PERSIST><<<launch_grid(init_table_kernel<COUNT, PERSIST>, g), g.nthr, g.smem,
                                            st>>>(d_jobs, d_job_start, n_jobs, g.tiles, g.queue, nh, census, rays,
                                                  out, d_work);
    else
        init_rows_kernel<COUNT, 4, PERSIST><<<launch_grid(init_rows_kernel<COUNT, 4, PERSIST>, g), g.nthr, g.smem,
                                              st>>>(d_jobs, d_job_start, n_jobs, g.tiles, g.queue, nh, census, rays,
                                                    out, d_work);
}
template <bool COUNT, bool PERSIST>
void pass_as(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g, uint64_t pass,
             float sig_inv, float sig_n, const uint64_t* census, const float2* rays, PlaneBuf prev, PlaneBuf next,
             unsigned long long* d_work, cudaStream_t st) {
    if (g.stream) {  // always persistent: block b owns slice b of the scratch
        if (!PERSIST) return;
        const int grid = std::min(launch_grid(pass_stream_kernel<COUNT, true>, g), g.scratch_blocks);
        pass_stream_kernel<COUNT, true><<<grid, STREAM_THREADS, stream_smem_bytes(), st>>>(
            d_jobs, d_job_start, n_jobs, g.tiles, g.queue, pass, sig_inv, sig_n, census, rays, prev, next, g.scratch,
            d_work);
        return;
    }
    if (g.tpp == SPLIT) {
        LaunchGeom gs = g;
        gs.nthr = split_threads(g.nthr);
        pass_split_kernel<COUNT, PERSIST><<<launch_grid(pass_split_kernel<COUNT, PERSIST>, gs), gs.nthr, gs.smem,
                                            st>>>(d_jobs, d_job_start, n_jobs, g.tiles, g.queue, pass, sig_inv, sig_n,
                                                  census, rays, prev, next, d_work);
        return;
    }
    pass_kernel<COUNT, 3, PERSIST><<<launch_grid(pass_kernel<COUNT, 3, PERSIST>, g), g.nthr, g.smem, st>>>(
        d_jobs, d_job_start, n_jobs, g.tiles, g.queue, pass, sig_inv, sig_n, census, rays, prev, next, d_work);
}
}  // namespace

cudaError_t launch_init(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g, int nh,
                        const uint64_t* census, const float2* rays, PlaneBuf out, unsigned long long* d_work,
                        cudaStream_t st, int variant) {
    if (g.tiles <= 0) return cudaSuccess;
    if (d_work) {
        if (g.queue)
            init_as<true, true>(variant, d_jobs, d_job_start, n_jobs, g, nh, census, rays, out, d_work, st);
        else
            init_as<true, false>(variant, d_jobs, d_job_start, n_jobs, g, nh, census, rays, out, d_work, st);
    } else {
        if (g.queue)
            init_as<false, true>(variant, d_jobs, d_job_start, n_jobs, g, nh, census, rays, out, nullptr, st);
        else
            init_as<false, false>(variant, d_jobs, d_job_start, n_jobs, g, nh, census, rays, out, nullptr, st);
    }
    return cudaGetLastError();
}

cudaError_t launch_pass(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g,
                        uint64_t pass, float sig_inv, float sig_n, const uint64_t* census, const float2* rays,
                        PlaneBuf prev, PlaneBuf next, unsigned long long* d_work, cudaStream_t st) {
    if (g.tiles <= 0) return cudaSuccess;
    if (g.stream && (!g.queue || !g.scratch || g.scratch_blocks <= 0)) return cudaErrorInvalidValue;
    if (d_work) {
        if (g.queue)
            pass_as<true, true>(d_jobs, d_job_start, n_jobs, g, pass, sig_inv, sig_n, census, rays, prev, next, d_work,
                                st);
        else
            pass_as<true, false>(d_jobs, d_job_start, n_jobs, g, pass, sig_inv, sig_n, census, rays, prev, next,
                                 d_work, st);
    } else {
        if (g.queue)
            pass_as<false, true>(d_jobs, d_job_start, n_jobs, g, pass, sig_inv, sig_n, census, rays, prev, next,
                                 nullptr, st);
        else
            pass_as<false, false>(d_jobs, d_job_start, n_jobs, g, pass, sig_inv, sig_n, census, rays, prev, next,
                                  nullptr, st);
    }
    return cudaGetLastError();
}

cudaError_t launch_init_learned(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g,
                                int nh, const uint64_t* census, const float2* rays, PlaneBuf out, const float* pred,
                                const int64_t* pred_off, float logit_thr, int n_local, float span, bool sweep_seeded,
                                unsigned long long* d_learned, cudaStream_t st) {
    if (g.tiles <= 0) return cudaSuccess;
    if (g.queue)
        init_learned_rows_kernel<true><<<launch_grid(init_learned_rows_kernel<true>, g), g.nthr, g.smem, st>>>(
            d_jobs, d_job_start, n_jobs, g.tiles, g.queue, nh, census, rays, out, pred, pred_off, logit_thr, n_local,
            span, (int)sweep_seeded, d_learned);
    else
        init_learned_rows_kernel<false><<<g.tiles, g.nthr, g.smem, st>>>(d_jobs, d_job_start, n_jobs, g.tiles,
                                                                          nullptr, nh, census, rays, out, pred,
                                                                          pred_off, logit_thr, n_local, span,
                                                                          (int)sweep_seeded, d_learned);
    return cudaGetLastError();
}

cudaError_t launch_gate(const DevJob* d_jobs, const int32_t* d_job_start, int n_jobs, const LaunchGeom& g,
                        float cost_thr, const uint64_t* census, PlaneBuf planes, float* depth, float* cost,
                        float* normal, cudaStream_t st) {
    if (g.tiles <= 0) return cudaSuccess;
    gate_kernel<<<g.tiles, g.nthr, 0, st>>>(d_jobs, d_job_start, n_jobs, cost_thr, census, planes, depth, cost,
                                            normal);
    return cudaGetLastError();
}

cudaError_t launch_cost_field(const DevJob* d_job, const int32_t* d_job_start, const LaunchGeom& g,
                              const uint64_t* census, const float2* rays, const float4* planes, const float* hints,
                              float* cost_out, int32_t* hsum_out, cudaStream_t st) {
    if (g.tiles <= 0) return cudaSuccess;
    cost_field_kernel<<<g.tiles, g.nthr, g.smem, st>>>(d_job, d_job_start, census, rays, planes, hints, cost_out,
                                                       hsum_out);
    return cudaGetLastError();
}

cudaError_t launch_f2i(const float* in, int n, int32_t* out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    f2i_kernel<<<(n + 255) / 256, 256, 0, st>>>(in, n, out);
    return cudaGetLastError();
}

}  // namespace rcmvs
