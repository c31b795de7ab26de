// census.cu — census transform + per-pixel rays for every view of a scene.
//
// census: mvs/src/lib.rs:119-142 (7x7, centre skipped, bit (dy+3)*7+(dx+3)
//   set iff the clamped neighbour is darker).  The reference compares
//   u8/255.0 in f32, a strictly monotone map, so comparing the u8 values
//   gives the same bits.
// rays:   mvs/src/stereo.rs:118-125 (Cam::normalize in f64, cast to f32;
//   sfm-lite/src/geom.rs:28-42).  IEEE f64 divide/multiply/add with FMA
//   contraction off reproduce the host's bits.
//
// One block = one 32x8 tile of one view; the grey tile plus a 3-pixel clamped
// halo is staged in shared memory.  HBM-bound: 1 B in, 16 B out per pixel.
#include "rcmvs_internal.cuh"

namespace rcmvs {

namespace {

constexpr int CTW = 32, CTH = 8, CH = 3;

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

__global__ void __launch_bounds__(CTW* CTH) census_rays_kernel(const DevView* __restrict__ views,
                                                             const int32_t* __restrict__ tile_start,
                                                             int n_views, const uint8_t* __restrict__ gray,
                                                             uint64_t* __restrict__ census,
                                                             float2* __restrict__ rays,
                                                             const double* __restrict__ cams) {
    __shared__ uint8_t tile[CTH + 2 * CH][CTW + 2 * CH + 2];
    const int v = find_item(tile_start, n_views, blockIdx.x);
    const DevView V = views[v];
    const int t = blockIdx.x - tile_start[v];
    const int tiles_x = (V.w + CTW - 1) / CTW;
    const int x0 = (t % tiles_x) * CTW, y0 = (t / tiles_x) * CTH;
    const uint8_t* g = gray + V.off;
    for (int i = threadIdx.x; i < (CTW + 2 * CH) * (CTH + 2 * CH); i += CTW * CTH) {
        int sx = i % (CTW + 2 * CH), sy = i / (CTW + 2 * CH);
        int gx = min(max(x0 - CH + sx, 0), V.w - 1);
        int gy = min(max(y0 - CH + sy, 0), V.h - 1);
        tile[sy][sx] = g[(size_t)gy * V.w + gx];
    }
    __syncthreads();
    const int lx = threadIdx.x % CTW, ly = threadIdx.x / CTW;
    const int x = x0 + lx, y = y0 + ly;
    if (x >= V.w || y >= V.h) return;
    const uint8_t c = tile[ly + CH][lx + CH];
    uint64_t bits = 0;
#pragma unroll
    for (int dy = -3; dy <= 3; ++dy)
#pragma unroll
        for (int dx = -3; dx <= 3; ++dx) {
            if (dx == 0 && dy == 0) continue;
            if (tile[ly + CH + dy][lx + CH + dx] < c) bits |= 1ull << ((dy + 3) * 7 + (dx + 3));
        }
    const size_t i = (size_t)V.off + (size_t)y * V.w + x;
    census[i] = bits;

    const double f = cams[4 * v], cx = cams[4 * v + 1], cy = cams[4 * v + 2], k = cams[4 * v + 3];
    const double u = (double)x, vv = (double)y;
    double xn = (u - cx) / f;
    double yn = (vv - cy) / f;
    for (int it = 0; it < 2; ++it) {
        double r2 = xn * xn + yn * yn;
        double d = 1.0 + k * r2;
        if (fabs(d) < 1e-12) break;
        xn = (u - cx) / (f * d);
        yn = (vv - cy) / (f * d);
    }
    rays[i] = make_float2((float)xn, (float)yn);
}

}  // namespace

cudaError_t launch_census_rays(const DevView* d_views, const int32_t* d_tile_start, int n_views,
                               int total_tiles, const uint8_t* gray, uint64_t* census, float2* rays,
                               const double* d_cams, cudaStream_t st) {
    if (total_tiles <= 0) return cudaSuccess;
    census_rays_kernel<<<total_tiles, CTW * CTH, 0, st>>>(d_views, d_tile_start, n_views, gray, census,
                                                          rays, d_cams);
    return cudaGetLastError();
}

}  // namespace rcmvs
