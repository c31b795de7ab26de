// fuse.cu — geometric-consistency fusion + voxel dedup on sm_100a.
//
// Restates mvs/src/fuse.rs:
//   sample_depth        fuse.rs:32-62    (device function sample_depth)
//   per-pixel check     fuse.rs:96-167   (candidates_kernel, one thread/pixel,
//                                          f64 as the reference)
//   voxel dedup         fuse.rs:176-214  (sort + in-order segmented sums)
//   PLY vertex records  fuse.rs:232-237  (reduce_kernel packs 15-byte records)
//
// The reference accumulates each voxel sequentially in view-then-pixel
// order.  Here candidates keep their global pixel index (views are
// concatenated in order), are compacted stably, keyed by the packed voxel
// index and radix-sorted stably, so each voxel's members stay in that order
// and one thread per voxel reproduces the reference's f64 sums bit for bit.
// Output order is the sorted key order (the reference's HashMap order is
// unspecified).
#include <thrust/iterator/counting_iterator.h>

#include <climits>
#include <cub/cub.cuh>

#include "rcmvs_internal.cuh"

namespace rcmvs {

namespace {

constexpr int FT = 256;  // threads per block for pixel kernels
constexpr int RT = 64;   // threads per block of the voxel reduce: few voxels, spread over every SM

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

// sfm-lite/src/geom.rs:28-42
__device__ __forceinline__ void cam_normalize(const FuseView& v, double u, double w, double& xn, double& yn) {
    xn = (u - v.cx) / v.f;
    yn = (w - v.cy) / v.f;
    // with k = 0 and a finite radius, d = 1 + 0 * r2 is exactly 1, f * d = f,
    // and both iterations give back xn, yn: skipped
    if (v.k == 0.0 && isfinite(xn * xn + yn * yn)) return;
    for (int it = 0; it < 2; ++it) {
        double r2 = xn * xn + yn * yn;
        double d = 1.0 + v.k * r2;
        if (fabs(d) < 1e-12) break;
        xn = (u - v.cx) / (v.f * d);
        yn = (w - v.cy) / (v.f * d);
    }
}

// nalgebra 3x3 products, k ascending
__device__ __forceinline__ void mat_vec(const double* m, const double* x, double* o) {
    for (int i = 0; i < 3; ++i) o[i] = m[3 * i] * x[0] + m[3 * i + 1] * x[1] + m[3 * i + 2] * x[2];
}
__device__ __forceinline__ void matt_vec(const double* m, const double* x, double* o) {
    for (int i = 0; i < 3; ++i) o[i] = m[i] * x[0] + m[3 + i] * x[1] + m[6 + i] * x[2];
}

// sfm-lite/src/geom.rs:64-75
__device__ __forceinline__ bool project(const FuseView& v, const double* x, double& u, double& w) {
    double xc[3];
    mat_vec(v.R, x, xc);
    for (int i = 0; i < 3; ++i) xc[i] = xc[i] + v.t[i];
    const double z = xc[2];
    if (z <= 1e-9) return false;
    const double xn = xc[0] / z, yn = xc[1] / z;
    const double r2 = xn * xn + yn * yn;
    const double d = 1.0 + v.k * r2;
    u = v.f * xn * d + v.cx;
    w = v.f * yn * d + v.cy;
    return true;
}

// Rust `f64 as i32` (saturating, NaN -> 0): cvt.rzi.s32.f64
__device__ __forceinline__ int f64_to_i32(double x) { return __double2int_rz(x); }

// fuse.rs:32-62
__device__ __forceinline__ double sample_depth(const float* __restrict__ dm, int w, int h, double u, double v) {
    const int u0 = f64_to_i32(floor(u));
    const int v0 = f64_to_i32(floor(v));
    // The reference tests `u0 + 1 >= w`.  u0 saturates at INT_MAX for points
    // barely in front of the camera, where `+ 1` would overflow (Rust wraps in
    // release builds and then panics on the slice index); `u0 >= w - 1` is
    // the same test without the overflow and treats such points as off-image.
    if (u0 < 0 || v0 < 0 || u0 >= w - 1 || v0 >= h - 1) return 0.0;
    const float fx = (float)(u - (double)u0);
    const float fy = (float)(v - (double)v0);
    const float d00 = __ldg(dm + (size_t)v0 * w + u0), d10 = __ldg(dm + (size_t)v0 * w + u0 + 1);
    const float d01 = __ldg(dm + (size_t)(v0 + 1) * w + u0), d11 = __ldg(dm + (size_t)(v0 + 1) * w + u0 + 1);
    const float ds[4] = {d00, d10, d01, d11};
    const float wt[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
    float acc = 0.f, wsum = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (ds[q] > 0.0f) {
            acc += ds[q] * wt[q];
            wsum += wt[q];
        }
    if (wsum > 1e-6f) return (double)(acc / wsum);
    return 0.0;
}

// Marks the pixels with a depth (z > 0) of the views that have a map; the
// consistency kernel then runs on the compacted list of these pixels only.
__global__ void __launch_bounds__(FT) valid_kernel(const FuseView* __restrict__ views,
                                                   const int32_t* __restrict__ blk_start,
                                                   const int32_t* __restrict__ blk_view, int n_items,
                                                   const float* __restrict__ depth, uint8_t* __restrict__ flag) {
    const int item = find_item(blk_start, n_items, blockIdx.x);
    const FuseView& v = views[blk_view[item]];
    const int64_t local = (int64_t)(blockIdx.x - blk_start[item]) * FT + threadIdx.x;
    if (local >= (int64_t)v.w * v.h) return;
    const size_t gi = (size_t)v.off + (size_t)local;
    flag[gi] = depth[gi] > 0.0f ? 1 : 0;
}

// fuse.rs:96-167 for one pixel with a depth: flag + averaged point.  One
// thread per entry of the list of such pixels (global indices; view k of
// the map-holding views starts at voff[k]).  Register cap 64 (four blocks
// per SM): on 100 1080p views it runs in 50 ms against 56 ms at 80
// registers, though it spills -- more resident warps hide the latency of
// the depth gathers from other views.
__global__ void __launch_bounds__(FT, 4) candidates_kernel(const FuseView* __restrict__ views,
                                                           const int64_t* __restrict__ voff,
                                                           const int32_t* __restrict__ vidx, int n_items,
                                                           const uint32_t* __restrict__ work, uint32_t n_work,
                                                           const int32_t* __restrict__ order,
                                                           const float* __restrict__ depth, uint32_t min_consistent,
                                                           double depth_diff, double reproj_px,
                                                           uint8_t* __restrict__ flag, double* __restrict__ pts) {
    const uint32_t t = blockIdx.x * FT + threadIdx.x;
    if (t >= n_work) return;
    const size_t gi = work[t];
    int lo = 0, hi = n_items - 1;  // the map-holding view that owns gi
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (voff[mid] <= (int64_t)gi)
            lo = mid;
        else
            hi = mid - 1;
    }
    const FuseView& v = views[vidx[lo]];
    const int64_t local = (int64_t)gi - v.off;
    const int px = (int)(local % v.w), py = (int)(local / v.w);
    const double zr = (double)depth[gi];
    uint8_t ok = 0;
    {
        double nx, ny;
        cam_normalize(v, (double)px, (double)py, nx, ny);
        const double xr[3] = {nx * zr, ny * zr, 1.0 * zr};
        const double dd[3] = {xr[0] - v.t[0], xr[1] - v.t[1], xr[2] - v.t[2]};
        double xw[3];
        matt_vec(v.R, dd, xw);
        double acc[3] = {xw[0], xw[1], xw[2]};
        uint32_t n_cons = 0;
        for (int q = v.order_begin; q < v.order_end; ++q) {
            const FuseView& sv = views[order[q]];
            double xs[3];
            mat_vec(sv.R, xw, xs);
            for (int a = 0; a < 3; ++a) xs[a] = xs[a] + sv.t[a];
            if (xs[2] <= 1e-6) continue;
            double us, vs;
            if (!project(sv, xw, us, vs)) continue;
            const double zs = sample_depth(depth + sv.off, sv.w, sv.h, us, vs);
            if (zs <= 0.0) continue;
            const double rel = fabs((xs[2] - zs) / xs[2]);
            if (rel < depth_diff) {
                double sx, sy;
                cam_normalize(sv, us, vs, sx, sy);
                const double xs2[3] = {sx * zs, sy * zs, 1.0 * zs};
                const double d2[3] = {xs2[0] - sv.t[0], xs2[1] - sv.t[1], xs2[2] - sv.t[2]};
                double xw2[3];
                matt_vec(sv.R, d2, xw2);
                if (reproj_px > 0.0) {  // extension: forward-backward reprojection gate
                    double ru, rv;
                    if (!project(v, xw2, ru, rv)) continue;
                    const double ex = ru - (double)px, ey = rv - (double)py;
                    if (!(sqrt(ex * ex + ey * ey) <= reproj_px)) continue;
                }
                for (int a = 0; a < 3; ++a) acc[a] += xw2[a];
                ++n_cons;
            }
        }
        if (n_cons >= min_consistent) {
            const double m = (double)(n_cons + 1);
            pts[3 * gi] = acc[0] / m;
            pts[3 * gi + 1] = acc[1] / m;
            pts[3 * gi + 2] = acc[2] / m;
            ok = 1;
        }
    }
    flag[gi] = ok;
}

// Rust `f64 as i64` (saturating, NaN -> 0): cvt.rzi.s64.f64
__device__ __forceinline__ long long vkey(double p, double cell) { return __double2ll_rz(floor(p / cell)); }

__global__ void keys_minmax_kernel(const uint32_t* __restrict__ cand, uint32_t n, const double* __restrict__ pts,
                                   double cell, long long* __restrict__ kmin, long long* __restrict__ kmax) {
    __shared__ long long smin[3][FT / 32], smax[3][FT / 32];
    long long lo[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, hi[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
    for (uint32_t c = blockIdx.x * FT + threadIdx.x; c < n; c += gridDim.x * FT) {
        const size_t g = cand[c];
        for (int a = 0; a < 3; ++a) {
            long long k = vkey(pts[3 * g + a], cell);
            lo[a] = min(lo[a], k);
            hi[a] = max(hi[a], k);
        }
    }
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = min(lo[a], __shfl_down_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_down_sync(0xffffffffu, hi[a], o));
        }
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) {
            smin[a][wid] = lo[a];
            smax[a][wid] = hi[a];
        }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int a = threadIdx.x;
        long long l = LLONG_MAX, h = LLONG_MIN;
        for (int q = 0; q < FT / 32; ++q) {
            l = min(l, smin[a][q]);
            h = max(h, smax[a][q]);
        }
        atomicMin(kmin + a, l);
        atomicMax(kmax + a, h);
    }
}

__global__ void pack_keys_kernel(const uint32_t* __restrict__ cand, uint32_t n, const double* __restrict__ pts,
                                 double cell, const long long* __restrict__ kmin, uint64_t* __restrict__ keys,
                                 uint32_t* __restrict__ vals) {
    const uint32_t c = blockIdx.x * FT + threadIdx.x;
    if (c >= n) return;
    const size_t g = cand[c];
    uint64_t key = 0;
    for (int a = 0; a < 3; ++a) {
        const uint64_t k = (uint64_t)(vkey(pts[3 * g + a], cell) - kmin[a]);
        key = (key << 21) | k;  // x in the high bits: lexicographic (x, y, z)
    }
    keys[c] = key;
    vals[c] = c;
}

// fuse.rs:194-213: in-order sums per voxel (u16 colour sums wrap), means,
// and the 15-byte PLY vertex record of fuse.rs:232-237.
__global__ void reduce_kernel(const uint32_t* __restrict__ run_off, const uint32_t* __restrict__ run_len,
                              const uint32_t* __restrict__ n_runs_p, const uint32_t* __restrict__ sorted_vals,
                              const uint32_t* __restrict__ cand, const double* __restrict__ pts,
                              const uint8_t* __restrict__ rgb, double* __restrict__ out_xyz,
                              uint8_t* __restrict__ out_rgb, uint8_t* __restrict__ ply) {
    const uint32_t r = blockIdx.x * RT + threadIdx.x;
    if (r >= *n_runs_p) return;
    const uint32_t b = run_off[r], n = run_len[r];
    double sx = 0.0, sy = 0.0, sz = 0.0;
    uint16_t cr = 0, cg = 0, cb = 0;
    // Members four at a time: the four chains of dependent loads (sorted
    // position -> candidate -> point) are issued together, then added in
    // member order, so the f64 sums are the sequential ones.
    constexpr int U = 4;
    uint32_t m = 0;
    for (; m + U <= n; m += U) {
        size_t g[U];
#pragma unroll
        for (int k = 0; k < U; ++k) g[k] = cand[sorted_vals[b + m + k]];
        double px[U], py[U], pz[U];
        uint8_t qr[U], qg[U], qb[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
            px[k] = pts[3 * g[k]];
            py[k] = pts[3 * g[k] + 1];
            pz[k] = pts[3 * g[k] + 2];
            qr[k] = rgb[3 * g[k]];
            qg[k] = rgb[3 * g[k] + 1];
            qb[k] = rgb[3 * g[k] + 2];
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
            sx += px[k];
            sy += py[k];
            sz += pz[k];
            cr = (uint16_t)(cr + qr[k]);
            cg = (uint16_t)(cg + qg[k]);
            cb = (uint16_t)(cb + qb[k]);
        }
    }
    for (; m < n; ++m) {
        const size_t g = cand[sorted_vals[b + m]];
        sx += pts[3 * g];
        sy += pts[3 * g + 1];
        sz += pts[3 * g + 2];
        cr = (uint16_t)(cr + rgb[3 * g]);
        cg = (uint16_t)(cg + rgb[3 * g + 1]);
        cb = (uint16_t)(cb + rgb[3 * g + 2]);
    }
    const double nn = (double)n;
    const double x = sx / nn, y = sy / nn, z = sz / nn;
    out_xyz[3 * (size_t)r] = x;
    out_xyz[3 * (size_t)r + 1] = y;
    out_xyz[3 * (size_t)r + 2] = z;
    uint8_t c3[3];
    const uint16_t cs[3] = {cr, cg, cb};
    for (int a = 0; a < 3; ++a) {
        double q = round((double)cs[a] / nn);  // half away from zero, as f64::round
        c3[a] = q <= 0.0 ? 0 : (q >= 255.0 ? 255 : (uint8_t)q);
        out_rgb[3 * (size_t)r + a] = c3[a];
    }
    if (ply) {
        const float fx = (float)x, fy = (float)y, fz = (float)z;
        uint8_t* o = ply + 15 * (size_t)r;
        const uint8_t* bx = reinterpret_cast<const uint8_t*>(&fx);
        const uint8_t* by = reinterpret_cast<const uint8_t*>(&fy);
        const uint8_t* bz = reinterpret_cast<const uint8_t*>(&fz);
        for (int q = 0; q < 4; ++q) {
            o[q] = bx[q];
            o[4 + q] = by[q];
            o[8 + q] = bz[q];
        }
        o[12] = c3[0];
        o[13] = c3[1];
        o[14] = c3[2];
    }
}

__global__ void init_minmax_kernel(long long* kmin, long long* kmax) {
    if (threadIdx.x < 3) {
        kmin[threadIdx.x] = LLONG_MAX;
        kmax[threadIdx.x] = LLONG_MIN;
    }
}

struct CountingIt {
    using value_type = uint32_t;
};

__global__ void iota_kernel(uint32_t* __restrict__ out, uint32_t n) {
    for (uint32_t i = blockIdx.x * FT + threadIdx.x; i < n; i += gridDim.x * FT) out[i] = i;
}

// Compacts the candidates' points and reference colours in list order.
__global__ void gather_cand_kernel(const uint32_t* __restrict__ cand, uint32_t n, const double* __restrict__ pts,
                                   const uint8_t* __restrict__ rgb, double* __restrict__ out_xyz,
                                   uint8_t* __restrict__ out_rgb) {
    for (uint32_t c = blockIdx.x * FT + threadIdx.x; c < n; c += gridDim.x * FT) {
        const size_t g = cand[c];
        for (int a = 0; a < 3; ++a) {
            out_xyz[3 * (size_t)c + a] = pts[3 * g + a];
            out_rgb[3 * (size_t)c + a] = rgb[3 * g + a];
        }
    }
}

}  // namespace

#define FCK(x)                                                                   \
    do {                                                                         \
        cudaError_t e_ = (x);                                                    \
        if (e_ != cudaSuccess) {                                                 \
            *err = std::string(#x) + ": " + cudaGetErrorString(e_);              \
            return RCMVS_E_CUDA;                                                 \
        }                                                                        \
    } while (0)

// Arena slots used by fusion (the stereo path uses slots below 16): 16-37
// and 70-74.
enum {
    S_FLAG = 16, S_PTS, S_CAND, S_NSEL, S_KMIN, S_KEYS, S_VALS, S_KEYS2, S_VALS2, S_RUNKEY, S_RUNLEN,
    S_RUNOFF, S_NRUNS, S_TEMP, S_OUTXYZ, S_OUTRGB, S_PLY, S_FVIEWS, S_ORDER, S_BLK, S_WORK, S_VOFF
};
enum { S_INXYZ = 70, S_INRGB, S_IOTA, S_GXYZ, S_GRGB };

unsigned fgrid(uint32_t n) { return (unsigned)std::max<uint32_t>(1, std::min<uint32_t>((n + FT - 1) / FT, 148u * 8u)); }

int fuse_candidates_device(DeviceArena& A, const FuseView* h_views, int n_views, const int32_t* h_order,
                           int n_order, const float* depth, uint32_t min_consistent, double depth_diff,
                           double reproj_px, const uint32_t** d_cand, uint32_t* n_cand_out, const double** d_pts,
                           cudaStream_t st, std::string* err, const SpanHook& hook) {
    // pixel-block table over the reference views that have a depth map
    std::vector<int32_t> blk_start, blk_view;
    int64_t total_blocks = 0, total_px = 0;
    for (int v = 0; v < n_views; ++v) {
        total_px = std::max<int64_t>(total_px, h_views[v].off + (int64_t)h_views[v].w * h_views[v].h);
        if (!h_views[v].has_depth || !h_views[v].is_ref) continue;
        blk_start.push_back((int32_t)total_blocks);
        blk_view.push_back(v);
        total_blocks += ((int64_t)h_views[v].w * h_views[v].h + FT - 1) / FT;
    }
    *n_cand_out = 0;
    *d_cand = nullptr;
    *d_pts = nullptr;
    if (blk_view.empty() || total_px == 0) return RCMVS_OK;
    if (total_blocks > INT32_MAX || total_px > (int64_t)UINT32_MAX) {
        *err = "fusion: scene too large for 32-bit candidate indices";
        return RCMVS_E_LIMIT;
    }
    const int n_items = (int)blk_view.size();
    blk_start.push_back((int32_t)total_blocks);
    void *p_views, *p_order, *p_blk, *p_flag, *p_pts;
    FCK(A.get(S_FVIEWS, sizeof(FuseView) * n_views, &p_views));
    FCK(A.get(S_ORDER, sizeof(int32_t) * std::max(1, n_order), &p_order));
    FCK(A.get(S_BLK, sizeof(int32_t) * (2 * n_items + 1), &p_blk));
    FCK(A.get(S_FLAG, (size_t)total_px, &p_flag));
    FCK(A.get(S_PTS, sizeof(double) * 3 * (size_t)total_px, &p_pts));
    FCK(cudaMemcpyAsync(p_views, h_views, sizeof(FuseView) * n_views, cudaMemcpyHostToDevice, st));
    if (n_order > 0) FCK(cudaMemcpyAsync(p_order, h_order, sizeof(int32_t) * n_order, cudaMemcpyHostToDevice, st));
    std::vector<int32_t> blk(blk_start);
    blk.insert(blk.end(), blk_view.begin(), blk_view.end());
    FCK(cudaMemcpyAsync(p_blk, blk.data(), sizeof(int32_t) * blk.size(), cudaMemcpyHostToDevice, st));
    uint8_t* flag = (uint8_t*)p_flag;
    double* pts = (double*)p_pts;
    // pixels of views without a depth map are never read: zero all flags
    FCK(cudaMemsetAsync(flag, 0, (size_t)total_px, st));
    const uint32_t npx = (uint32_t)total_px;
    void *p_cand, *p_nsel, *p_temp, *p_work, *p_voff;
    FCK(A.get(S_CAND, sizeof(uint32_t) * npx, &p_cand));
    FCK(A.get(S_WORK, sizeof(uint32_t) * npx, &p_work));
    FCK(A.get(S_NSEL, sizeof(uint32_t) * 4, &p_nsel));
    FCK(A.get(S_VOFF, sizeof(int64_t) * n_items, &p_voff));
    std::vector<int64_t> voff(n_items);
    for (int k = 0; k < n_items; ++k) voff[k] = h_views[blk_view[k]].off;
    FCK(cudaMemcpyAsync(p_voff, voff.data(), sizeof(int64_t) * n_items, cudaMemcpyHostToDevice, st));
    thrust::counting_iterator<uint32_t> it(0);
    size_t tb = 0;
    FCK(cub::DeviceSelect::Flagged(nullptr, tb, it, flag, (uint32_t*)p_cand, (uint32_t*)p_nsel, npx, st));
    FCK(A.get(S_TEMP, tb, &p_temp));
    hook.begin("fuse_candidates");
    // the pixels with a depth, compacted, then one thread each
    valid_kernel<<<(unsigned)total_blocks, FT, 0, st>>>((const FuseView*)p_views, (const int32_t*)p_blk,
                                                       (const int32_t*)p_blk + n_items + 1, n_items, depth, flag);
    FCK(cudaGetLastError());
    FCK(cub::DeviceSelect::Flagged(p_temp, tb, it, flag, (uint32_t*)p_work, (uint32_t*)p_nsel + 1, npx, st));
    uint32_t n_work = 0;
    FCK(cudaMemcpyAsync(&n_work, (uint32_t*)p_nsel + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    if (n_work > 0)
        candidates_kernel<<<(n_work + FT - 1) / FT, FT, 0, st>>>(
            (const FuseView*)p_views, (const int64_t*)p_voff, (const int32_t*)p_blk + n_items + 1, n_items,
            (const uint32_t*)p_work, n_work, (const int32_t*)p_order, depth, min_consistent, depth_diff, reproj_px,
            flag, pts);
    FCK(cudaGetLastError());
    hook.end("fuse_candidates");

    // stable compaction of candidate pixel indices (view-then-pixel order)
    FCK(cub::DeviceSelect::Flagged(p_temp, tb, it, flag, (uint32_t*)p_cand, (uint32_t*)p_nsel, npx, st));
    uint32_t n_cand = 0;
    FCK(cudaMemcpyAsync(&n_cand, p_nsel, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    *n_cand_out = n_cand;
    *d_cand = (const uint32_t*)p_cand;
    *d_pts = pts;
    return RCMVS_OK;
}

int fuse_reduce_device(DeviceArena& A, const uint32_t* d_cand, uint32_t n_cand, const double* pts,
                       const uint8_t* rgb, double cell, double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply,
                       uint64_t* n_points, cudaStream_t st, std::string* err, const SpanHook& hook) {
    *n_points = 0;
    if (n_cand == 0) return RCMVS_OK;
    const void* p_cand = d_cand;
    void* p_temp;
    size_t tb = 0;
    // voxel keys, packed 21 bits per axis
    void* p_kmin;
    FCK(A.get(S_KMIN, sizeof(long long) * 6, &p_kmin));
    long long* kmin = (long long*)p_kmin;
    long long* kmax = kmin + 3;
    init_minmax_kernel<<<1, 32, 0, st>>>(kmin, kmax);
    const unsigned gb = (unsigned)std::min<uint32_t>((n_cand + FT - 1) / FT, 148u * 8u);
    keys_minmax_kernel<<<gb, FT, 0, st>>>((const uint32_t*)p_cand, n_cand, pts, cell, kmin, kmax);
    FCK(cudaGetLastError());
    long long hk[6];
    FCK(cudaMemcpyAsync(hk, kmin, sizeof(hk), cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    for (int a = 0; a < 3; ++a) {
        unsigned long long span = (unsigned long long)(hk[3 + a] - hk[a]);
        if (hk[3 + a] < hk[a] || span >= (1ull << 21)) {
            *err = "fusion: voxel index range exceeds 2^21 cells per axis (cell too small for the cloud)";
            return RCMVS_E_LIMIT;
        }
    }
    void *p_keys, *p_vals, *p_keys2, *p_vals2;
    FCK(A.get(S_KEYS, sizeof(uint64_t) * n_cand, &p_keys));
    FCK(A.get(S_VALS, sizeof(uint32_t) * n_cand, &p_vals));
    FCK(A.get(S_KEYS2, sizeof(uint64_t) * n_cand, &p_keys2));
    FCK(A.get(S_VALS2, sizeof(uint32_t) * n_cand, &p_vals2));
    pack_keys_kernel<<<(n_cand + FT - 1) / FT, FT, 0, st>>>((const uint32_t*)p_cand, n_cand, pts, cell, kmin,
                                                            (uint64_t*)p_keys, (uint32_t*)p_vals);
    FCK(cudaGetLastError());
    // stable LSD radix sort over the 63 used bits
    tb = 0;
    FCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint64_t*)p_keys, (uint64_t*)p_keys2,
                                        (const uint32_t*)p_vals, (uint32_t*)p_vals2, n_cand, 0, 63, st));
    FCK(A.get(S_TEMP, tb, &p_temp));
    FCK(cub::DeviceRadixSort::SortPairs(p_temp, tb, (const uint64_t*)p_keys, (uint64_t*)p_keys2,
                                        (const uint32_t*)p_vals, (uint32_t*)p_vals2, n_cand, 0, 63, st));
    // runs of equal keys = voxels
    void *p_runkey, *p_runlen, *p_runoff, *p_nruns;
    FCK(A.get(S_RUNKEY, sizeof(uint64_t) * n_cand, &p_runkey));
    FCK(A.get(S_RUNLEN, sizeof(uint32_t) * n_cand, &p_runlen));
    FCK(A.get(S_RUNOFF, sizeof(uint32_t) * n_cand, &p_runoff));
    FCK(A.get(S_NRUNS, sizeof(uint32_t) * 4, &p_nruns));
    tb = 0;
    FCK(cub::DeviceRunLengthEncode::Encode(nullptr, tb, (const uint64_t*)p_keys2, (uint64_t*)p_runkey,
                                           (uint32_t*)p_runlen, (uint32_t*)p_nruns, n_cand, st));
    size_t tb2 = 0;
    FCK(cub::DeviceScan::ExclusiveSum(nullptr, tb2, (const uint32_t*)p_runlen, (uint32_t*)p_runoff, n_cand, st));
    FCK(A.get(S_TEMP, std::max(tb, tb2), &p_temp));
    FCK(cub::DeviceRunLengthEncode::Encode(p_temp, tb, (const uint64_t*)p_keys2, (uint64_t*)p_runkey,
                                           (uint32_t*)p_runlen, (uint32_t*)p_nruns, n_cand, st));
    uint32_t n_runs = 0;
    FCK(cudaMemcpyAsync(&n_runs, p_nruns, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    FCK(cub::DeviceScan::ExclusiveSum(p_temp, tb2, (const uint32_t*)p_runlen, (uint32_t*)p_runoff, n_runs, st));
    void *p_oxyz, *p_orgb, *p_ply;
    FCK(A.get(S_OUTXYZ, sizeof(double) * 3 * n_runs, &p_oxyz));
    FCK(A.get(S_OUTRGB, 3 * (size_t)n_runs, &p_orgb));
    FCK(A.get(S_PLY, 15 * (size_t)n_runs, &p_ply));
    hook.begin("fuse_reduce");
    reduce_kernel<<<(n_runs + RT - 1) / RT, RT, 0, st>>>((const uint32_t*)p_runoff, (const uint32_t*)p_runlen,
                                                         (const uint32_t*)p_nruns, (const uint32_t*)p_vals2,
                                                         (const uint32_t*)p_cand, pts, rgb, (double*)p_oxyz,
                                                         (uint8_t*)p_orgb, (uint8_t*)p_ply);
    FCK(cudaGetLastError());
    hook.end("fuse_reduce");
    *d_xyz = (double*)p_oxyz;
    *d_rgb = (uint8_t*)p_orgb;
    *d_ply = (uint8_t*)p_ply;
    *n_points = n_runs;
    return RCMVS_OK;
}

int fuse_reduce_host(DeviceArena& A, const double* h_xyz, const uint8_t* h_rgb, uint64_t n, double cell,
                     double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply, uint64_t* n_points, cudaStream_t st,
                     std::string* err, const SpanHook& hook) {
    *n_points = 0;
    if (n == 0) return RCMVS_OK;
    if (n > (uint64_t)UINT32_MAX) {
        *err = "fusion: more than 2^32 candidates";
        return RCMVS_E_LIMIT;
    }
    void *p_xyz, *p_rgb, *p_iota;
    FCK(A.get(S_INXYZ, sizeof(double) * 3 * n, &p_xyz));
    FCK(A.get(S_INRGB, 3 * n, &p_rgb));
    FCK(A.get(S_IOTA, sizeof(uint32_t) * n, &p_iota));
    FCK(cudaMemcpyAsync(p_xyz, h_xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    FCK(cudaMemcpyAsync(p_rgb, h_rgb, 3 * n, cudaMemcpyHostToDevice, st));
    iota_kernel<<<fgrid((uint32_t)n), FT, 0, st>>>((uint32_t*)p_iota, (uint32_t)n);
    FCK(cudaGetLastError());
    return fuse_reduce_device(A, (const uint32_t*)p_iota, (uint32_t)n, (const double*)p_xyz, (const uint8_t*)p_rgb,
                              cell, d_xyz, d_rgb, d_ply, n_points, st, err, hook);
}

int fuse_reduce_devptr(DeviceArena& A, const double* d_in_xyz, const uint8_t* d_in_rgb, uint64_t n, double cell,
                       double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply, uint64_t* n_points, cudaStream_t st,
                       std::string* err, const SpanHook& hook) {
    *n_points = 0;
    if (n == 0) return RCMVS_OK;
    if (n > (uint64_t)UINT32_MAX) {
        *err = "fusion: more than 2^32 candidates";
        return RCMVS_E_LIMIT;
    }
    void* p_iota;
    FCK(A.get(S_IOTA, sizeof(uint32_t) * n, &p_iota));
    iota_kernel<<<fgrid((uint32_t)n), FT, 0, st>>>((uint32_t*)p_iota, (uint32_t)n);
    FCK(cudaGetLastError());
    return fuse_reduce_device(A, (const uint32_t*)p_iota, (uint32_t)n, d_in_xyz, d_in_rgb, cell, d_xyz, d_rgb, d_ply,
                              n_points, st, err, hook);
}

int fuse_gather_device(DeviceArena& A, const uint32_t* d_cand, uint32_t n, const double* pts, const uint8_t* rgb,
                       double** d_xyz, uint8_t** d_rgb, cudaStream_t st, std::string* err) {
    void *p_xyz, *p_rgb;
    FCK(A.get(S_GXYZ, sizeof(double) * 3 * std::max<uint32_t>(n, 1), &p_xyz));
    FCK(A.get(S_GRGB, 3 * (size_t)std::max<uint32_t>(n, 1), &p_rgb));
    if (n > 0) {
        gather_cand_kernel<<<fgrid(n), FT, 0, st>>>(d_cand, n, pts, rgb, (double*)p_xyz, (uint8_t*)p_rgb);
        FCK(cudaGetLastError());
    }
    *d_xyz = (double*)p_xyz;
    *d_rgb = (uint8_t*)p_rgb;
    return RCMVS_OK;
}

int fuse_device(DeviceArena& A, const FuseView* h_views, int n_views, const int32_t* h_order, int n_order,
                const float* depth, const uint8_t* rgb, double cell, uint32_t min_consistent, double depth_diff,
                double reproj_px, double** d_xyz, uint8_t** d_rgb, uint8_t** d_ply, FuseResult* res,
                cudaStream_t st, std::string* err, const SpanHook& hook) {
    res->n_candidates = res->n_points = 0;
    const uint32_t* cand = nullptr;
    const double* pts = nullptr;
    uint32_t n_cand = 0;
    int rc = fuse_candidates_device(A, h_views, n_views, h_order, n_order, depth, min_consistent, depth_diff,
                                    reproj_px, &cand, &n_cand, &pts, st, err, hook);
    if (rc) return rc;
    res->n_candidates = n_cand;
    return fuse_reduce_device(A, cand, n_cand, pts, rgb, cell, d_xyz, d_rgb, d_ply, &res->n_points, st, err, hook);
}

}  // namespace rcmvs
