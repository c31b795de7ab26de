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
// One block = one 128x8 tile of one view, 256 threads; a thread owns 4
// horizontally adjacent pixels.  The grey tile plus a clamped halo (3 rows,
// 4 columns) is staged in shared memory as 32-bit words, so a thread reads
// each window row of its 4 pixels as three words.  The 48 comparisons are
// made for the 4 pixels at once, one byte lane each (SIMD within a 32-bit
// register: an unsigned per-byte less-than from one subtraction that cannot
// borrow across bytes and one three-input logic op), and accumulated in
// "byte planes" (plane P, byte p holds census bits 8P..8P+7 of pixel p),
// which a byte permute turns into the 4 census words.  Census and rays leave
// as 16-byte stores.  HBM-bound by design: 1 B in, 16 B out per pixel.
#include "rcmvs_internal.cuh"

namespace rcmvs {

namespace {

constexpr int CPX = 4;                     // pixels per thread (along x)
constexpr int CTW = 32 * CPX, CTH = 8;     // tile: a warp covers 128 columns of one row
constexpr int CHY = 3;                     // halo rows above and below
constexpr int CWORDS = (CTW + 8) / 4;      // staged words per row: columns x0-4 .. x0+CTW+3
constexpr int CSROWS = CTH + 2 * CHY;      // staged rows

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

// Bit 7 of each byte of the result is set iff that byte of a is less than
// the byte of c (unsigned).  cl = c & 0x7f7f7f7f.  (a | 0x80) - (c & 0x7f)
// lies in [1, 255] per byte, so the subtraction never borrows across bytes,
// and its bit 7 says whether a's low 7 bits are >= c's; a >= c holds when
// a's top bit is set and c's is not, or the top bits agree and the low bits
// compare >=.
__device__ __forceinline__ uint32_t bytes_lt(uint32_t a, uint32_t c, uint32_t cl) {
    const uint32_t t = (a | 0x80808080u) - cl;
    const uint32_t ge = (a & ~c) | (~(a ^ c) & t);
    return ~ge;
}

// Cam::normalize's two fixed-point iterations (geom.rs:28-42), f64.
__device__ __forceinline__ void undistort(double u, double v, double f, double cx, double cy, double k, double& xn,
                                          double& yn) {
    for (int it = 0; it < 2; ++it) {
        const double r2 = xn * xn + yn * yn;
        const double d = 1.0 + k * r2;
        if (fabs(d) < 1e-12) break;
        xn = (u - cx) / (f * d);
        yn = (v - cy) / (f * d);
    }
}

__global__ void __launch_bounds__(32 * CTH) census_rays_kernel(const DevView* __restrict__ views,
                                                              const int32_t* __restrict__ tile_start,
                                                              int n_views, const uint8_t* __restrict__ gray,
                                                              uint64_t* __restrict__ census,
                                                              float2* __restrict__ rays,
                                                              const double* __restrict__ cams) {
    __shared__ uint32_t tile[CSROWS][CWORDS];
    const int v = find_item(tile_start, n_views, blockIdx.x);
    const DevView V = views[v];
    const int t = blockIdx.x - tile_start[v];
    const int tiles_x = (V.w + CTW - 1) / CTW;
    const int x0 = (t % tiles_x) * CTW, y0 = (t / tiles_x) * CTH;
    const uint8_t* g = gray + V.off;
    // stage: word c of row r holds columns x0-4+4c .. x0-4+4c+3 (clamped)
    for (int i = threadIdx.x; i < CSROWS * CWORDS; i += 32 * CTH) {
        const int r = i / CWORDS, c = i % CWORDS;
        const int gy = min(max(y0 - CHY + r, 0), V.h - 1);
        const uint8_t* row = g + (size_t)gy * V.w;
        const int gx = x0 - 4 + 4 * c;
        uint32_t wd = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) wd |= (uint32_t)__ldg(row + min(max(gx + b, 0), V.w - 1)) << (8 * b);
        tile[r][c] = wd;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
    const int xb = x0 + CPX * lane, y = y0 + wy;
    if (xb >= V.w || y >= V.h) return;

    // the 4 centres, one per byte, from the window's middle row
    const uint32_t cw = tile[wy + CHY][lane + 1];
    const uint32_t cl = cw & 0x7f7f7f7fu;
    uint32_t plane[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int dy = -3; dy <= 3; ++dy) {
        const uint32_t* row = tile[wy + CHY + dy];
        const uint32_t w0 = row[lane], w1 = row[lane + 1], w2 = row[lane + 2];
#pragma unroll
        for (int dx = -3; dx <= 3; ++dx) {
            if (dx == 0 && dy == 0) continue;
            // bytes 4+dx .. 7+dx of (w0, w1, w2): neighbour (dx, dy) of each pixel
            const int s = 4 + dx;  // 1..7
            const uint32_t a = s < 4 ? __funnelshift_r(w0, w1, 8 * s)
                                     : (s == 4 ? w1 : __funnelshift_r(w1, w2, 8 * (s - 4)));
            const uint32_t lt = bytes_lt(a, cw, cl);
            const int k = (dy + 3) * 7 + (dx + 3);  // census bit
            const int q = k & 7;
            plane[k >> 3] |= (lt >> (7 - q)) & (0x01010101u << q);
        }
    }
    const size_t i0 = (size_t)V.off + (size_t)y * V.w + xb;
    const int n = min(CPX, V.w - xb);
    uint64_t cen[CPX];
#pragma unroll
    for (int p = 0; p < CPX; ++p) {
        const uint32_t sel = (uint32_t)p | ((uint32_t)(p + 4) << 4);  // byte p of x, byte p of y
        const uint32_t lo = __byte_perm(__byte_perm(plane[0], plane[1], sel), __byte_perm(plane[2], plane[3], sel),
                                        0x5410);
        const uint32_t hi =
            __byte_perm(__byte_perm(plane[4], plane[5], sel), plane[6], 0x4410 | (p << 8)) & 0x00ffffffu;
        cen[p] = ((uint64_t)hi << 32) | lo;
    }

    const double f = cams[4 * v], cx = cams[4 * v + 1], cy = cams[4 * v + 2], k = cams[4 * v + 3];
    const double vv = (double)y;
    const double yn0 = (vv - cy) / f;
    float2 ray[CPX];
#pragma unroll
    for (int p = 0; p < CPX; ++p) {
        const double u = (double)(xb + p);
        double xn = (u - cx) / f;
        double yn = yn0;
        // with k = 0 and a finite radius, d = 1 + 0*r2 is exactly 1, f*d = f,
        // and the iterations reproduce xn, yn: skipped
        if (!(k == 0.0 && isfinite(xn * xn + yn * yn))) undistort(u, vv, f, cx, cy, k, xn, yn);
        ray[p] = make_float2((float)xn, (float)yn);
    }
    if (n == CPX && (i0 & 1) == 0) {
        ulonglong2* cd = reinterpret_cast<ulonglong2*>(census + i0);
        cd[0] = make_ulonglong2(cen[0], cen[1]);
        cd[1] = make_ulonglong2(cen[2], cen[3]);
        float4* rd = reinterpret_cast<float4*>(rays + i0);
        rd[0] = make_float4(ray[0].x, ray[0].y, ray[1].x, ray[1].y);
        rd[1] = make_float4(ray[2].x, ray[2].y, ray[3].x, ray[3].y);
    } else {
#pragma unroll
        for (int p = 0; p < CPX; ++p)
            if (p < n) {
                census[i0 + p] = cen[p];
                rays[i0 + p] = ray[p];
            }
    }
}

}  // namespace

int census_tiles(int w, int h) { return ((w + CTW - 1) / CTW) * ((h + CTH - 1) / CTH); }

cudaError_t launch_census_rays(const DevView* d_views, const int32_t* d_tile_start, int n_views,
                               int total_tiles, const uint8_t* gray, uint64_t* census, float2* rays,
                               const double* d_cams, cudaStream_t st) {
    if (total_tiles <= 0) return cudaSuccess;
    census_rays_kernel<<<total_tiles, 32 * CTH, 0, st>>>(d_views, d_tile_start, n_views, gray, census, rays,
                                                         d_cams);
    return cudaGetLastError();
}

}  // namespace rcmvs
