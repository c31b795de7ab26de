// sift.cu — SIFT feature extraction on sm_100a.
//
// Restates sfm-lite/src/sift.rs (extract_sift, :435-555) for one image:
//
//   resize      load-time resize to max_dim (resize.cu; `.max(1)` sides)
//   pyramid     per octave six Gaussian levels (separable f32 blur with
//               clamped edges, f64 kernel weights cast to f32, taps summed in
//               order: sift.rs:51-93), five DoGs, 2x2 box downsample of
//               level 3 for the next octave (sift.rs:95-134)
//   extrema     one thread per (DoG level 1-3, pixel): the 24-neighbour test,
//               the quadratic fit (nalgebra's cofactor 3x3 inverse, f64), the
//               contrast and curvature tests (sift.rs:176-262); flags are
//               compacted stably, so keypoints keep the reference's
//               (octave, level, y, x) order; each octave's count stays on the
//               device and the next octave starts without waiting for it
//   orientation one warp per keypoint (in response order, see output):
//               lanes evaluate 32 window samples at a time (atan2, exp in
//               f64), each lane owns histogram bins and
//               adds the samples that fall in them in window order, so every
//               bin is the reference's sequential f64 sum; lane 0 smooths and
//               picks up to four peaks (sift.rs:274-334)
//   descriptor  one warp per (keypoint, peak): the same split over the window
//               (bilinear gradients, rotation, trilinear weights; up to 8
//               histogram entries per sample).  Lane L owns the 4 bins of cell
//               column L / 8 and orientation L % 8, so it finds its share of a
//               sample from the sample's (row, column, orientation) base by
//               arithmetic; L2 -> clip 0.2 -> L2 in f32 (sift.rs:340-431)
//   output      the reference sorts its descriptors by response (stable) and
//               keeps the first max_features (sift.rs:543-544).  A descriptor's
//               response is its keypoint's, so that order is the keypoints of
//               all octaves sorted stably by response (CUB radix sort) with
//               each keypoint's peaks in turn; orientations, pairs and
//               descriptors are produced in that order until max_features
//               valid ones exist -- the same output without the orientations
//               and descriptors the cap would discard (about 2k of 27k
//               keypoints at 1600x1200)
//
// The library builds with --fmad=false: every f32/f64 product and sum rounds
// as written, so the pyramid, the DoGs and the extrema with their fitted
// positions and responses are those of the CPU restatement bit for bit.  Orientation and
// descriptor use the device's f64 exp / atan2 / sin / cos, which may differ
// from the host libm in the last bit; their results agree with the CPU
// restatement to a tolerance, and a histogram bin or peak decision at an exact boundary can
// differ.
#include <thrust/iterator/counting_iterator.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <cub/cub.cuh>
#include <string>
#include <vector>

#include "ctx_internal.cuh"

namespace rcmvs {

namespace {

constexpr int NSPO = 3;
constexpr int NLEV = NSPO + 3;  // blurred levels per octave
constexpr int NDOG = NSPO + 2;
constexpr int DESC_LEN = 128;
constexpr int MAX_TAPS = 32;
constexpr double SIGMA0 = 1.6;
constexpr double ASSUMED_BLUR = 0.5;
constexpr double EDGE_THR = 10.0;
constexpr double PI = 3.14159265358979323846;
constexpr int WARPS = 4;  // warps per block in the keypoint kernels

struct BlurTaps {
    int radius;
    float k[MAX_TAPS];
};

struct KpArrays {  // raw keypoints in the reference's (octave, level, y, x) order
    double* x;       // octave coordinates
    double* y;
    double* resp;
    int32_t* level;
    int32_t* oct;
};

constexpr int MAX_OCT = 8;
struct OctTable {  // per octave: gradients of DoG levels 1..NSPO, size, scale
    const float* gx[MAX_OCT];
    const float* gy[MAX_OCT];
    int w[MAX_OCT], h[MAX_OCT];
    double scale[MAX_OCT];
};

__device__ __host__ __forceinline__ double level_sigma(int l) {
    return SIGMA0 * (double)(1 << (int)((double)l / (double)NSPO));
}

__global__ void to_float_kernel(const uint8_t* __restrict__ g, int64_t n, float* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)g[i] / 255.0f;
}

// sift.rs:65-77 (horizontal) and :79-90 (vertical)
template <bool VERT>
__global__ void blur_kernel(const float* __restrict__ src, float* __restrict__ dst, int w, int h,
                            const __grid_constant__ BlurTaps taps) {
    const int64_t n = (int64_t)w * h;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / w), x = (int)(i - (int64_t)y * w);
        float acc = 0.0f;
        for (int ki = 0; ki <= 2 * taps.radius; ++ki) {
            if (VERT) {
                const int yy = min(max(y + ki - taps.radius, 0), h - 1);
                acc = acc + taps.k[ki] * src[(int64_t)yy * w + x];
            } else {
                const int xx = min(max(x + ki - taps.radius, 0), w - 1);
                acc = acc + taps.k[ki] * src[(int64_t)y * w + xx];
            }
        }
        dst[i] = acc;
    }
}

__global__ void dog_kernel(const float* __restrict__ lev, float* __restrict__ dog, int64_t npx) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
        for (int d = 0; d < NDOG; ++d) dog[d * npx + i] = lev[(d + 1) * npx + i] - lev[d * npx + i];
}

// sift.rs:95-110
__global__ void downsample_kernel(const float* __restrict__ src, int w, int h, float* __restrict__ dst, int nw,
                                  int nh) {
    const int64_t n = (int64_t)nw * nh;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / nw), x = (int)(i - (int64_t)y * nw);
        const int x0 = min(2 * x, w - 1), y0 = min(2 * y, h - 1);
        const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
        const float s = src[(int64_t)y0 * w + x0] + src[(int64_t)y0 * w + x1] + src[(int64_t)y1 * w + x0] +
                        src[(int64_t)y1 * w + x1];
        dst[i] = 0.25f * s;
    }
}

// sift.rs:137-149, for levels 1..NSPO
__global__ void grad_kernel(const float* __restrict__ lev, int w, int h, float* __restrict__ gx,
                            float* __restrict__ gy) {
    const int64_t npx = (int64_t)w * h;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < NSPO * npx;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int l = (int)(t / npx);
        const int64_t i = t - (int64_t)l * npx;
        const int y = (int)(i / w), x = (int)(i - (int64_t)y * w);
        const float* img = lev + (l + 1) * npx;
        float a = 0.0f, b = 0.0f;
        if (x >= 1 && y >= 1 && x + 1 < w && y + 1 < h) {
            a = img[i + 1] - img[i - 1];
            b = img[i + w] - img[i - w];
        }
        gx[t] = a;
        gy[t] = b;
    }
}

// nalgebra 0.32 Matrix3::try_inverse: cofactors over the determinant
__device__ __forceinline__ bool inverse3(const double m[9], double o[9]) {
    const double m11 = m[0], m12 = m[1], m13 = m[2], m21 = m[3], m22 = m[4], m23 = m[5], m31 = m[6], m32 = m[7],
                 m33 = m[8];
    const double a = m22 * m33 - m32 * m23;
    const double b = m21 * m33 - m31 * m23;
    const double c = m21 * m32 - m31 * m22;
    const double det = m11 * a - m12 * b + m13 * c;
    if (det == 0.0) return false;
    o[0] = a / det;
    o[1] = (m13 * m32 - m33 * m12) / det;
    o[2] = (m12 * m23 - m22 * m13) / det;
    o[3] = -b / det;
    o[4] = (m11 * m33 - m31 * m13) / det;
    o[5] = (m13 * m21 - m23 * m11) / det;
    o[6] = c / det;
    o[7] = (m12 * m31 - m32 * m11) / det;
    o[8] = (m11 * m22 - m21 * m12) / det;
    return true;
}

// sift.rs:176-262.  Thread t = (level - 1) * npx + pixel.
__global__ void extrema_kernel(const float* __restrict__ dogs, int w, int h, double thr, uint8_t* __restrict__ flag,
                               double* __restrict__ kx, double* __restrict__ ky, double* __restrict__ kresp) {
    const int64_t npx = (int64_t)w * h;
    const double edge_lim = (EDGE_THR + 1.0) * (EDGE_THR + 1.0) / EDGE_THR;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < NSPO * npx;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int level = 1 + (int)(t / npx);
        const int64_t i = t - (int64_t)(level - 1) * npx;
        const int y = (int)(i / w), x = (int)(i - (int64_t)y * w);
        uint8_t ok = 0;
        if (x >= 1 && y >= 1 && x + 1 < w && y + 1 < h) {
            const float* dog = dogs + level * npx;
            const float* below = dogs + (level - 1) * npx;
            const float* above = dogs + (level + 1) * npx;
            const float v = dog[i];
            if (!((double)fabsf(v) < thr)) {
                bool is_max = true, is_min = true;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dy == 0 && dx == 0) continue;
                        const int64_t j = i + (int64_t)dy * w + dx;
                        const float n0 = dog[j], n1 = below[j], n2 = above[j];
                        if (n0 >= v || n1 >= v || n2 >= v) is_max = false;
                        if (n0 <= v || n1 <= v || n2 <= v) is_min = false;
                    }
                if (is_max || is_min) {
                    const float fdx = 0.5f * (dog[i + 1] - dog[i - 1]);
                    const float fdy = 0.5f * (dog[i + w] - dog[i - w]);
                    const float fds = 0.5f * (above[i] - below[i]);
                    const float dxx = dog[i + 1] + dog[i - 1] - 2.0f * v;
                    const float dyy = dog[i + w] + dog[i - w] - 2.0f * v;
                    const float dss = above[i] + below[i] - 2.0f * v;
                    const float dxy = 0.25f * (dog[i + w + 1] + dog[i - w - 1] - dog[i + w - 1] - dog[i - w + 1]);
                    const float dxs = 0.25f * (above[i + 1] + below[i - 1] - above[i - 1] - below[i + 1]);
                    const float dys = 0.25f * (above[i + w] + below[i - w] - above[i - w] - below[i + w]);
                    const double hm[9] = {dxx, dxy, dxs, dxy, dyy, dys, dxs, dys, dss};
                    double hi[9];
                    if (inverse3(hm, hi)) {
                        const double g0 = -(double)fdx, g1 = -(double)fdy, g2 = -(double)fds;
                        const double ox = hi[0] * g0 + hi[1] * g1 + hi[2] * g2;
                        const double oy = hi[3] * g0 + hi[4] * g1 + hi[5] * g2;
                        const double os = hi[6] * g0 + hi[7] * g1 + hi[8] * g2;
                        if (!(fabs(ox) > 1.0 || fabs(oy) > 1.0 || fabs(os) > 1.0)) {
                            const double contrast =
                                (double)v + 0.5 * ((double)fdx * ox + (double)fdy * oy + (double)fds * os);
                            const double tr = (double)(dxx + dyy);
                            const double det = (double)(dxx * dyy - dxy * dxy);
                            if (!(fabs(contrast) < thr) && !(det <= 0.0 || tr * tr / det > edge_lim)) {
                                ok = 1;
                                kx[t] = (double)x + ox;
                                ky[t] = (double)y + oy;
                                kresp[t] = fabs(contrast);
                            }
                        }
                    }
                }
            }
        }
        flag[t] = ok;
    }
}

// Appends the compacted keypoints of one octave (sel: indices into its flag
// space; counts[o]: each octave's count, on the device) after those of the
// octaves before it.
__global__ void gather_kp_kernel(const uint32_t* __restrict__ sel, const int* __restrict__ counts, int octave,
                                 int64_t npx, const double* __restrict__ kx, const double* __restrict__ ky,
                                 const double* __restrict__ kresp, KpArrays kp) {
    int64_t base = 0;
    for (int q = 0; q < octave; ++q) base += counts[q];
    const int n = counts[octave];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t t = sel[k];
        kp.x[base + k] = kx[t];
        kp.y[base + k] = ky[t];
        kp.resp[base + k] = kresp[t];
        kp.level[base + k] = 1 + (int)((int64_t)t / npx);
        kp.oct[base + k] = octave;
    }
}

__device__ __forceinline__ double rem_euclid(double a, double b) {
    const double r = fmod(a, b);
    return r < 0.0 ? r + fabs(b) : r;
}

// sift.rs:274-334.  One warp per keypoint, for the keypoints at sorted
// positions base .. base + n - 1 (skp[pos] = keypoint); theta[4 pos ..] and
// cnt[pos] (0 when the keypoint is outside the 8-pixel margin of the image,
// sift.rs:519-521).
__global__ void __launch_bounds__(32 * WARPS) orient_kernel(KpArrays kp, const uint32_t* __restrict__ skp,
                                                           int64_t base, int n, const __grid_constant__ OctTable oct,
                                                           int img_w, int img_h, double* __restrict__ theta,
                                                           int32_t* __restrict__ cnt) {
    __shared__ int sbin[WARPS][32];
    __shared__ double sval[WARPS][32];
    __shared__ double shist[WARPS][36];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * WARPS + wid;
    if (i >= n) return;
    const int64_t k = base + i;  // output position
    const uint32_t kk = skp[k];
    const double kx = kp.x[kk], ky = kp.y[kk];
    const int level = kp.level[kk], o = kp.oct[kk];
    const double scale = oct.scale[o];
    const double x0 = kx * scale, y0 = ky * scale;
    if (x0 < 8.0 || y0 < 8.0 || x0 >= (double)img_w - 8.0 || y0 >= (double)img_h - 8.0) {
        if (lane == 0) cnt[k] = 0;
        return;
    }
    const int w = oct.w[o], h = oct.h[o];
    const int64_t npx = (int64_t)w * h;
    const float* gx = oct.gx[o] + (level - 1) * npx;
    const float* gy = oct.gy[o] + (level - 1) * npx;
    const double sigma = 1.5 * level_sigma(level);
    const int radius = (int)fmax(ceil(3.0 * sigma), 1.0);
    const double s2 = 2.0 * sigma * sigma;
    const long long xr = (long long)round(kx), yr = (long long)round(ky);
    const int side = 2 * radius + 1, total = side * side;
    const int b0 = lane, b1 = lane + 32;
    double acc0 = 0.0, acc1 = 0.0;
    for (int base = 0; base < total; base += 32) {
        const int s = base + lane;
        int bin = -1;
        double val = 0.0;
        if (s < total) {
            const int dy = s / side - radius, dx = s % side - radius;
            const long long sx = xr + dx, sy = yr + dy;
            if (!(sx < 1 || sy < 1 || sx >= w - 1 || sy >= h - 1)) {
                const int64_t i = sy * w + sx;
                const float a = gx[i], b = gy[i];
                const double mag = sqrt((double)(a * a + b * b));
                const double ang = atan2((double)b, (double)a);
                const double wgt = exp((-((double)dx * (double)dx) - (double)dy * (double)dy) / s2);
                const double fb = floor((ang + PI) / (2.0 * PI) * 36.0);
                bin = !(fb > 0.0) ? 0 : (int)((long long)fb % 36);
                val = wgt * mag;
            }
        }
        sbin[wid][lane] = bin;
        sval[wid][lane] = val;
        __syncwarp();
        const int m = min(32, total - base);
        for (int t = 0; t < m; ++t) {
            const int b = sbin[wid][t];
            if (b == b0)
                acc0 += sval[wid][t];
            else if (b == b1)
                acc1 += sval[wid][t];
        }
        __syncwarp();
    }
    shist[wid][b0] = acc0;
    if (b1 < 36) shist[wid][b1] = acc1;
    __syncwarp();
    if (lane == 0) {
        double hist[36];
        for (int b = 0; b < 36; ++b) hist[b] = shist[wid][b];
        for (int it = 0; it < 2; ++it) {
            double sm[36];
            for (int b = 0; b < 36; ++b) sm[b] = (hist[(b + 35) % 36] + 2.0 * hist[b] + hist[(b + 1) % 36]) / 4.0;
            for (int b = 0; b < 36; ++b) hist[b] = sm[b];
        }
        double maxv = 0.0;
        for (int b = 0; b < 36; ++b) maxv = fmax(maxv, hist[b]);
        int np = 0;
        if (maxv < 1e-12) {
            theta[4 * (int64_t)k] = 0.0;
            np = 1;
        } else {
            const double thresh = 0.8 * maxv;
            for (int b = 0; b < 36 && np < 4; ++b) {
                const double prev = hist[(b + 35) % 36], next = hist[(b + 1) % 36];
                if (hist[b] > prev && hist[b] > next && hist[b] >= thresh) {
                    const double denom = hist[b] * 2.0 - prev - next;
                    const double d = fabs(denom) > 1e-12 ? 0.5 * (prev - next) / denom : 0.0;
                    const double th = ((double)b + d) / 36.0 * 2.0 * PI - PI;
                    theta[4 * (int64_t)k + np++] = rem_euclid(th, 2.0 * PI);
                }
            }
            if (np == 0) theta[4 * (int64_t)k + np++] = 0.0;
        }
        cnt[k] = np;
    }
}

// (keypoint, peak) pairs of the keypoints at sorted positions base ..
// base + n - 1, peaks in order, appended at pair index at + off[i] + p.
__global__ void pairs_kernel(const uint32_t* __restrict__ skp, int64_t base, int n, const int32_t* __restrict__ cnt,
                             const int32_t* __restrict__ off, const double* __restrict__ theta, int64_t at,
                             int32_t* __restrict__ pair_kp, double* __restrict__ pair_theta) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int64_t pos = base + i;
        for (int p = 0; p < cnt[pos]; ++p) {
            pair_kp[at + off[i] + p] = (int32_t)skp[pos];
            pair_theta[at + off[i] + p] = theta[4 * pos + p];
        }
    }
}

__global__ void iota_kernel(uint32_t* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)i;
}

// sift.rs:151-166
__device__ __forceinline__ float bilinear(const float* __restrict__ img, int w, int h, double x, double y) {
    const long long x0 = (long long)floor(x), y0 = (long long)floor(y);
    const float fx = (float)(x - (double)x0), fy = (float)(y - (double)y0);
    const long long xm = w - 1, ym = h - 1;
    const long long ax = min(max(x0, 0LL), xm), ay = min(max(y0, 0LL), ym);
    const long long bx = min(max(x0 + 1, 0LL), xm), by = min(max(y0 + 1, 0LL), ym);
    const float a = img[ay * w + ax] * (1.0f - fx) + img[ay * w + bx] * fx;
    const float b = img[by * w + ax] * (1.0f - fx) + img[by * w + bx] * fx;
    return a * (1.0f - fy) + b * fy;
}

// sift.rs:340-431.  One warp per (keypoint, peak) pair, for the pairs
// base .. base + n_pairs - 1 (in output order); descriptor and validity
// stored at the pair's index.
__global__ void __launch_bounds__(32 * WARPS) desc_kernel(KpArrays kp, int64_t base, int n_pairs,
                                                         const int32_t* __restrict__ pair_kp,
                                                         const double* __restrict__ pair_theta,
                                                         const __grid_constant__ OctTable oct,
                                                         float* __restrict__ desc, uint8_t* __restrict__ valid) {
    constexpr int D = 4, N = 8;
    __shared__ int hdr[WARPS][32];  // per sample: packed (by0, bx0, ob0 mod 8), or -1
    __shared__ double cv[WARPS][32 * 8];
    __shared__ float sd[WARPS][DESC_LEN];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * WARPS + wid;
    if (i >= n_pairs) return;
    const int64_t pos = base + i;
    const int k = pair_kp[pos];
    const double x = kp.x[k], y = kp.y[k], th = pair_theta[pos];
    const int level = kp.level[k], o = kp.oct[k];
    const int w = oct.w[o], h = oct.h[o];
    const int64_t npx = (int64_t)w * h;
    const float* gxi = oct.gx[o] + (level - 1) * npx;
    const float* gyi = oct.gy[o] + (level - 1) * npx;
    const double sigma = level_sigma(level);
    const double cell = 3.0 * sigma;
    const int radius = (int)ceil(sqrt(1.5) * cell * ((double)D + 1.0) * 0.5);
    const double cos_t = cos(th), sin_t = sin(th);
    const double exp_scale = -1.0 / ((double)(D * D) * 0.5);
    const double half = (double)D * 0.5;
    const int side = 2 * radius + 1, total = side * side;
    // Lane L owns the bins 32q + L (q = 0..3): cell row q, cell column L / 8,
    // orientation L % 8.  A sample adds to such a bin at most once.
    const int cx = lane >> 3, co = lane & 7;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int base = 0; base < total; base += 32) {
        const int s = base + lane;
        int hd = -1;
        if (s < total) {
            const int dy = s / side - radius, dx = s % side - radius;
            const double sx = x + (double)dx, sy = y + (double)dy;
            if (!(sx < 1.0 || sy < 1.0 || sx >= (double)w - 2.0 || sy >= (double)h - 2.0)) {
                const double gx = (double)bilinear(gxi, w, h, sx, sy);
                const double gy = (double)bilinear(gyi, w, h, sx, sy);
                const double mag = sqrt(gx * gx + gy * gy);
                if (!(mag < 1e-12)) {
                    const double rx = cos_t * (double)dx + sin_t * (double)dy;
                    const double ry = -sin_t * (double)dx + cos_t * (double)dy;
                    const double bx = rx / cell + half - 0.5;
                    const double by = ry / cell + half - 0.5;
                    if (!(bx < -1.0 || by < -1.0 || bx > (double)D || by > (double)D)) {
                        const double ang = atan2(gy, gx) - th;
                        const double ob = rem_euclid(ang, 2.0 * PI) / (2.0 * PI) * (double)N;
                        double wgt =
                            ((bx - half + 0.5) * (bx - half + 0.5) + (by - half + 0.5) * (by - half + 0.5)) * exp_scale;
                        wgt = exp(wgt) * mag;
                        // bx, by in [-1, 4], ob in [0, 8]
                        const int bx0 = (int)floor(bx), by0 = (int)floor(by), ob0 = (int)floor(ob);
                        const double fx = bx - (double)bx0, fy = by - (double)by0, fo = ob - (double)ob0;
#pragma unroll
                        for (int iy = 0; iy < 2; ++iy)
#pragma unroll
                            for (int ix = 0; ix < 2; ++ix) {
                                const double wy = iy == 0 ? 1.0 - fy : fy;
                                const double wx = ix == 0 ? 1.0 - fx : fx;
#pragma unroll
                                for (int io = 0; io < 2; ++io) {
                                    const double wo = io == 0 ? 1.0 - fo : fo;
                                    cv[wid][lane * 8 + iy * 4 + ix * 2 + io] = wgt * wx * wy * wo;
                                }
                            }
                        hd = ((by0 + 2) << 8) | ((bx0 + 2) << 4) | (ob0 & 7);
                    }
                }
            }
        }
        hdr[wid][lane] = hd;
        __syncwarp();
        const int m = min(32, total - base);
        for (int t = 0; t < m; ++t) {
            const int hv = hdr[wid][t];
            if (hv < 0) continue;
            const int ix = cx - (((hv >> 4) & 15) - 2);
            const int io = (co - (hv & 7)) & 7;
            if ((unsigned)ix > 1u || io > 1) continue;
            const int by0 = (hv >> 8) - 2;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int iy = q - by0;
                if (iy == 0 || iy == 1) acc[q] += cv[wid][t * 8 + iy * 4 + ix * 2 + io];
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) sd[wid][lane + 32 * q] = (float)acc[q];
    __syncwarp();
    if (lane == 0) {
        float* d = sd[wid];
        float ss = 0.0f;
        for (int i = 0; i < DESC_LEN; ++i) ss = ss + d[i] * d[i];
        const float norm = sqrtf(ss);
        bool ok = !(norm < 1e-6f);
        if (ok) {
            for (int i = 0; i < DESC_LEN; ++i) d[i] = d[i] / norm;
            for (int i = 0; i < DESC_LEN; ++i)
                if (d[i] > 0.2f) d[i] = 0.2f;
            float ss2 = 0.0f;
            for (int i = 0; i < DESC_LEN; ++i) ss2 = ss2 + d[i] * d[i];
            const float norm2 = sqrtf(ss2);
            ok = !(norm2 < 1e-6f);
            if (ok)
                for (int i = 0; i < DESC_LEN; ++i) d[i] = d[i] / norm2;
        }
        valid[pos] = ok ? 1 : 0;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) desc[pos * DESC_LEN + lane + 32 * q] = sd[wid][lane + 32 * q];
}

// sift.rs:543-554: output i is the sorted position sel[i] (the i-th valid
// descriptor in response order); clamped position, descriptor, colour.
__global__ void final_kernel(const uint32_t* __restrict__ sel, int n, const int32_t* __restrict__ pair_kp, KpArrays kp,
                             const __grid_constant__ OctTable oct,
                             const float* __restrict__ desc, const uint8_t* __restrict__ rgb, int w, int h,
                             double* __restrict__ pts, float* __restrict__ odesc, uint8_t* __restrict__ col) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (wid >= n) return;
    const uint32_t pos = sel[wid];
    if (lane == 0) {
        const int k = pair_kp[pos];
        const double scale = oct.scale[kp.oct[k]];
        const double x = fmin(fmax(kp.x[k] * scale, 0.0), (double)(w - 1));
        const double y = fmin(fmax(kp.y[k] * scale, 0.0), (double)(h - 1));
        const long long px = min((long long)round(x), (long long)(w - 1));
        const long long py = min((long long)round(y), (long long)(h - 1));
        pts[2 * wid] = x;
        pts[2 * wid + 1] = y;
        for (int c = 0; c < 3; ++c) col[3 * wid + c] = rgb[3 * (py * w + px) + c];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
        odesc[(int64_t)wid * DESC_LEN + lane + 32 * q] = desc[(int64_t)pos * DESC_LEN + lane + 32 * q];
}

unsigned grid_of(int64_t n, int threads = 256) {
    const int64_t b = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

// sift.rs:51-63: f64 kernel weights, normalised, cast to f32 per tap
bool blur_taps(double sigma, BlurTaps& t) {
    const int radius = (int)std::max(std::ceil(sigma * 3.0), 1.0);
    if (2 * radius + 1 > MAX_TAPS) return false;
    std::vector<double> k(2 * radius + 1);
    const double s2 = 2.0 * sigma * sigma;
    double sum = 0.0;
    for (int i = 0; i < 2 * radius + 1; ++i) {
        const double x = (double)i - (double)radius;
        k[i] = std::exp(-x * x / s2);
        sum += k[i];
    }
    t.radius = radius;
    for (int i = 0; i < 2 * radius + 1; ++i) t.k[i] = (float)(k[i] / sum);
    return true;
}

int sfail(rcmvs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

#define SCK(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return sfail(ctx, e_ == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,    \
                         std::string(#x) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

// Context arena slots 80-159.
enum {
    F_IN = 80, F_GRAY, F_RGB, F_BASE, F_LEV, F_TMP, F_DOG, F_FLAG, F_KX, F_KY, F_KRESP, F_SEL, F_NSEL, F_TEMP,
    F_KPX, F_KPY, F_KPRESP, F_KPLEV, F_KPOCT, F_THETA, F_CNT, F_OFF, F_PKP, F_PTH, F_PIDX, F_SRESP, F_SIDX,
    F_DESC, F_VALID, F_OSEL, F_PTS, F_FDESC, F_COL, F_NEXT, F_OCTCNT,
    F_GRAD = 130  // 130 + 2 * octave: gx, + 1: gy (octaves 0..7)
};

// Grows an arena slot to `need` bytes keeping its first `keep` bytes: a
// device-to-device copy into a buffer of twice the need when the slot is too
// small, else the slot as it is.
int grow_copy(rcmvs_ctx* ctx, int slot, size_t need, size_t keep, void** p) {
    DeviceArena& A = ctx->arena;
    if ((int)A.slots.size() <= slot) A.slots.resize(slot + 1);
    DeviceArena::Slot& s = A.slots[slot];
    if (s.p && s.bytes >= need) {
        *p = s.p;
        return RCMVS_OK;
    }
    void* np_ = nullptr;
    const size_t cap = std::max<size_t>(2 * need, 1 << 20);
    SCK(cudaMalloc(&np_, cap));
    if (keep && s.p) SCK(cudaMemcpyAsync(np_, s.p, keep, cudaMemcpyDeviceToDevice, ctx->stream));
    SCK(cudaStreamSynchronize(ctx->stream));
    if (s.p) SCK(cudaFree(s.p));
    s.p = np_;
    s.bytes = cap;
    *p = np_;
    return RCMVS_OK;
}

}  // namespace
}  // namespace rcmvs

using namespace rcmvs;

extern "C" {

void rcmvs_sift_options_default(rcmvs_sift_options* o) {
    if (!o) return;
    o->max_dim = 1600;  // sift.rs:28-31
    o->max_features = 2048;
    o->reserved = 0;
    o->reserved2 = 0;
    o->contrast_thr = 0.0067;
}

void rcmvs_sift_frame_free(rcmvs_sift_frame* f) {
    if (!f) return;
    std::free(f->pts);
    std::free(f->desc);
    std::free(f->colors);
    f->pts = nullptr;
    f->desc = nullptr;
    f->colors = nullptr;
    f->n = 0;
}

int rcmvs_extract_sift(rcmvs_ctx* ctx, const uint8_t* img, int32_t w0, int32_t h0, int32_t channels,
                       const rcmvs_sift_options* opts, rcmvs_sift_frame* out) {
    if (!ctx || !img || !opts || !out) return sfail(ctx, RCMVS_E_ARG, "rcmvs_extract_sift: bad argument");
    std::memset(out, 0, sizeof(*out));
    // sift.rs:436-444: resize so the long side is at most max_dim (sides >= 1)
    int32_t w = w0, h = h0;
    const int32_t m = std::max(w0, h0);
    if (m > 0 && (uint32_t)m > opts->max_dim) {
        const double s = (double)opts->max_dim / (double)m;
        w = (int32_t)std::max(std::round((double)w0 * s), 1.0);
        h = (int32_t)std::max(std::round((double)h0 * s), 1.0);
    }
    int rc = resize_check(ctx, w0, h0, channels, w, h);
    if (rc) return rc;
    SCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    DeviceArena& A = ctx->arena;
    const int64_t n_in = (int64_t)w0 * h0, npx0 = (int64_t)w * h;
    void *p_in, *p_gray, *p_rgb, *p_base;
    SCK(A.get(F_IN, (size_t)n_in * channels, &p_in));
    SCK(A.get(F_GRAY, (size_t)npx0, &p_gray));
    SCK(A.get(F_RGB, 3 * (size_t)npx0, &p_rgb));
    SCK(A.get(F_BASE, sizeof(float) * (size_t)npx0, &p_base));
    SCK(cudaMemcpyAsync(p_in, img, (size_t)n_in * channels, cudaMemcpyHostToDevice, st));
    const int* d_err = nullptr;
    rc = resize_device(ctx, (const uint8_t*)p_in, w0, h0, channels, w, h, (uint8_t*)p_gray, (uint8_t*)p_rgb, &d_err);
    if (rc) return rc;
    to_float_kernel<<<grid_of(npx0), 256, 0, st>>>((const uint8_t*)p_gray, npx0, (float*)p_base);
    SCK(cudaGetLastError());

    int n_oct = 1;  // sift.rs:458-461
    while ((std::max(w, h) >> n_oct) >= 40 && n_oct < 8) ++n_oct;
    BlurTaps first{}, inc[NLEV];
    const double fs = std::sqrt(std::max(SIGMA0 * SIGMA0 - ASSUMED_BLUR * ASSUMED_BLUR, 1e-4));
    if (!blur_taps(fs, first)) return sfail(ctx, RCMVS_E_LIMIT, "sift: blur kernel too wide");
    for (int l = 1; l < NLEV; ++l) {
        const double sp = level_sigma(l - 1), sc = level_sigma(l);
        if (!blur_taps(std::sqrt(std::max(sc * sc - sp * sp, 1e-4)), inc[l]))
            return sfail(ctx, RCMVS_E_LIMIT, "sift: blur kernel too wide");
    }

    const SpanHook& hook = ctx->hook();
    if (n_oct > MAX_OCT) return sfail(ctx, RCMVS_E_LIMIT, "sift: too many octaves");
    OctTable table{};
    int ow = w, oh = h;
    thrust::counting_iterator<uint32_t> it(0);
    void *p_temp, *p_nsel, *p_octcnt;
    SCK(A.get(F_NSEL, sizeof(int) * 4, &p_nsel));
    SCK(A.get(F_OCTCNT, sizeof(int) * MAX_OCT, &p_octcnt));
    int* d_oct = (int*)p_octcnt;
    // keypoint arrays sized for every pixel of DoG levels 1-3 of every
    // octave, so the octaves run back to back with their counts on the device
    int64_t kcap = 0;
    for (int o = 0, tw = w, th = h; o < n_oct; ++o, tw = std::max(tw / 2, 1), th = std::max(th / 2, 1))
        kcap += NSPO * (int64_t)tw * th;
    KpArrays kp{};
    {
        void *p_x, *p_y, *p_r, *p_l, *p_o;
        SCK(A.get(F_KPX, 8 * (size_t)kcap, &p_x));
        SCK(A.get(F_KPY, 8 * (size_t)kcap, &p_y));
        SCK(A.get(F_KPRESP, 8 * (size_t)kcap, &p_r));
        SCK(A.get(F_KPLEV, 4 * (size_t)kcap, &p_l));
        SCK(A.get(F_KPOCT, 4 * (size_t)kcap, &p_o));
        kp = KpArrays{(double*)p_x, (double*)p_y, (double*)p_r, (int32_t*)p_l, (int32_t*)p_o};
    }
    for (int o = 0; o < n_oct; ++o) {
        const int64_t npx = (int64_t)ow * oh;
        void *p_lev, *p_tmp, *p_dog, *p_flag, *p_kx, *p_ky, *p_kr, *p_sel;
        SCK(A.get(F_LEV, sizeof(float) * NLEV * (size_t)npx, &p_lev));
        SCK(A.get(F_TMP, sizeof(float) * (size_t)npx, &p_tmp));
        SCK(A.get(F_DOG, sizeof(float) * NDOG * (size_t)npx, &p_dog));
        float* lev = (float*)p_lev;
        float* tmp = (float*)p_tmp;
        // level 0: the base (blurred by the first sigma in octave 0)
        const float* base = (const float*)p_base;
        hook.begin("sift_pyramid");
        if (o == 0) {
            blur_kernel<false><<<grid_of(npx), 256, 0, st>>>(base, tmp, ow, oh, first);
            blur_kernel<true><<<grid_of(npx), 256, 0, st>>>(tmp, lev, ow, oh, first);
        } else {
            SCK(cudaMemcpyAsync(lev, base, sizeof(float) * npx, cudaMemcpyDeviceToDevice, st));
        }
        for (int l = 1; l < NLEV; ++l) {
            blur_kernel<false><<<grid_of(npx), 256, 0, st>>>(lev + (l - 1) * npx, tmp, ow, oh, inc[l]);
            blur_kernel<true><<<grid_of(npx), 256, 0, st>>>(tmp, lev + l * npx, ow, oh, inc[l]);
        }
        SCK(cudaGetLastError());
        dog_kernel<<<grid_of(npx), 256, 0, st>>>(lev, (float*)p_dog, npx);
        SCK(cudaGetLastError());
        hook.end("sift_pyramid");
        const int64_t nt = NSPO * npx;
        if (nt > (int64_t)UINT32_MAX) return sfail(ctx, RCMVS_E_LIMIT, "sift: octave too large");
        SCK(A.get(F_FLAG, (size_t)nt, &p_flag));
        SCK(A.get(F_KX, sizeof(double) * (size_t)nt, &p_kx));
        SCK(A.get(F_KY, sizeof(double) * (size_t)nt, &p_ky));
        SCK(A.get(F_KRESP, sizeof(double) * (size_t)nt, &p_kr));
        SCK(A.get(F_SEL, sizeof(uint32_t) * (size_t)nt, &p_sel));
        hook.begin("sift_extrema");
        extrema_kernel<<<grid_of(nt), 256, 0, st>>>((const float*)p_dog, ow, oh, opts->contrast_thr,
                                                     (uint8_t*)p_flag, (double*)p_kx, (double*)p_ky, (double*)p_kr);
        SCK(cudaGetLastError());
        hook.end("sift_extrema");
        size_t tb = 0;
        SCK(cub::DeviceSelect::Flagged(nullptr, tb, it, (const uint8_t*)p_flag, (uint32_t*)p_sel, d_oct + o,
                                       (int)nt, st));
        SCK(A.get(F_TEMP, tb, &p_temp));
        SCK(cub::DeviceSelect::Flagged(p_temp, tb, it, (const uint8_t*)p_flag, (uint32_t*)p_sel, d_oct + o,
                                       (int)nt, st));
        table.w[o] = ow;
        table.h[o] = oh;
        table.scale[o] = std::pow(2.0, o);
        gather_kp_kernel<<<grid_of(nt), 256, 0, st>>>((const uint32_t*)p_sel, d_oct, o, npx, (const double*)p_kx,
                                                       (const double*)p_ky, (const double*)p_kr, kp);
        SCK(cudaGetLastError());
        void *p_gx, *p_gy;
        SCK(A.get(F_GRAD + 2 * o, sizeof(float) * NSPO * (size_t)npx, &p_gx));
        SCK(A.get(F_GRAD + 2 * o + 1, sizeof(float) * NSPO * (size_t)npx, &p_gy));
        table.gx[o] = (const float*)p_gx;
        table.gy[o] = (const float*)p_gy;
        grad_kernel<<<grid_of(NSPO * npx), 256, 0, st>>>(lev, ow, oh, (float*)p_gx, (float*)p_gy);
        SCK(cudaGetLastError());
        // next octave's base: level NSPO downsampled 2x2 (sift.rs:488-492)
        const int nw = std::max(ow / 2, 1), nh = std::max(oh / 2, 1);
        if (o + 1 < n_oct) {
            void* p_next;
            SCK(A.get(F_NEXT, sizeof(float) * (size_t)nw * nh, &p_next));
            downsample_kernel<<<grid_of((int64_t)nw * nh), 256, 0, st>>>(lev + NSPO * npx, ow, oh, (float*)p_next,
                                                                         nw, nh);
            SCK(cudaGetLastError());
            SCK(A.get(F_BASE, sizeof(float) * (size_t)nw * nh, &p_base));
            SCK(cudaMemcpyAsync(p_base, p_next, sizeof(float) * (size_t)nw * nh, cudaMemcpyDeviceToDevice, st));
        }
        ow = nw;
        oh = nh;
    }
    int bad = 0;
    int oc[MAX_OCT] = {0};
    if (d_err) SCK(cudaMemcpyAsync(&bad, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(oc, d_oct, sizeof(int) * n_oct, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (bad) return sfail(ctx, RCMVS_E_CUDA, "sift: resize tap table overflow");
    int64_t nkp = 0;  // keypoints of all octaves
    for (int o = 0; o < n_oct; ++o) nkp += oc[o];
    const uint64_t n_raw = (uint64_t)nkp;
    if (nkp > INT32_MAX / 4) return sfail(ctx, RCMVS_E_LIMIT, "sift: too many keypoints");

    // The reference computes every (keypoint, peak) descriptor in (octave,
    // keypoint, peak) order, sorts them by their keypoint's response with a
    // stable sort and keeps the first max_features (sift.rs:497-544).  The
    // same order is the keypoints sorted stably by response with each one's
    // peaks in turn, so keypoints are sorted first and orientations, pairs
    // and descriptors are produced in that order until max_features valid
    // descriptors exist (a descriptor that normalises to nothing is dropped,
    // as in the reference).
    const int64_t cap = (int64_t)opts->max_features;
    int64_t kdone = 0, np = 0, done = 0, n_valid = 0;
    void *p_kidx = nullptr, *p_sresp = nullptr, *p_skp = nullptr, *p_th = nullptr, *p_cnt = nullptr,
         *p_off = nullptr, *p_pkp = nullptr, *p_pth = nullptr, *p_desc = nullptr, *p_valid = nullptr,
         *p_osel = nullptr;
    if (nkp > 0 && cap > 0) {
        SCK(A.get(F_PIDX, sizeof(uint32_t) * (size_t)nkp, &p_kidx));
        SCK(A.get(F_SRESP, sizeof(double) * (size_t)nkp, &p_sresp));
        SCK(A.get(F_SIDX, sizeof(uint32_t) * (size_t)nkp, &p_skp));
        SCK(A.get(F_THETA, sizeof(double) * 4 * (size_t)nkp, &p_th));
        SCK(A.get(F_CNT, sizeof(int32_t) * (size_t)nkp, &p_cnt));
        SCK(A.get(F_OFF, sizeof(int32_t) * (size_t)nkp, &p_off));
        SCK(A.get(F_PKP, sizeof(int32_t) * 4 * (size_t)nkp, &p_pkp));
        SCK(A.get(F_PTH, sizeof(double) * 4 * (size_t)nkp, &p_pth));
        SCK(A.get(F_VALID, 4 * (size_t)nkp, &p_valid));
        SCK(A.get(F_OSEL, sizeof(uint32_t) * 4 * (size_t)nkp, &p_osel));
        iota_kernel<<<grid_of(nkp), 256, 0, st>>>((uint32_t*)p_kidx, nkp);
        SCK(cudaGetLastError());
        size_t tb = 0;
        SCK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, (const double*)kp.resp, (double*)p_sresp,
                                                      (const uint32_t*)p_kidx, (uint32_t*)p_skp, (int)nkp, 0, 64,
                                                      st));
        SCK(A.get(F_TEMP, tb, &p_temp));
        SCK(cub::DeviceRadixSort::SortPairsDescending(p_temp, tb, (const double*)kp.resp, (double*)p_sresp,
                                                      (const uint32_t*)p_kidx, (uint32_t*)p_skp, (int)nkp, 0, 64,
                                                      st));
    }
    while (n_valid < cap && (done < np || kdone < nkp)) {
        if (done == np) {
            // orientations of the next keypoints in response order, and their pairs
            const int64_t ck = std::min<int64_t>(nkp - kdone, std::max<int64_t>(cap - n_valid, 64));
            hook.begin("sift_orient");
            orient_kernel<<<(unsigned)((ck + WARPS - 1) / WARPS), 32 * WARPS, 0, st>>>(
                kp, (const uint32_t*)p_skp, kdone, (int)ck, table, w, h, (double*)p_th, (int32_t*)p_cnt);
            SCK(cudaGetLastError());
            hook.end("sift_orient");
            size_t tb = 0;
            SCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, (const int32_t*)p_cnt + kdone, (int32_t*)p_off, (int)ck,
                                              st));
            SCK(A.get(F_TEMP, tb, &p_temp));
            SCK(cub::DeviceScan::ExclusiveSum(p_temp, tb, (const int32_t*)p_cnt + kdone, (int32_t*)p_off, (int)ck,
                                              st));
            pairs_kernel<<<grid_of(ck), 256, 0, st>>>((const uint32_t*)p_skp, kdone, (int)ck, (const int32_t*)p_cnt,
                                                      (const int32_t*)p_off, (const double*)p_th, np,
                                                      (int32_t*)p_pkp, (double*)p_pth);
            SCK(cudaGetLastError());
            int last_off = 0, last_cnt = 0;
            SCK(cudaMemcpyAsync(&last_off, (int32_t*)p_off + ck - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            SCK(cudaMemcpyAsync(&last_cnt, (int32_t*)p_cnt + kdone + ck - 1, sizeof(int), cudaMemcpyDeviceToHost,
                                st));
            SCK(cudaStreamSynchronize(st));
            kdone += ck;
            np += (int64_t)last_off + last_cnt;
            continue;
        }
        const int64_t chunk = std::min<int64_t>(np - done, std::max<int64_t>(cap - n_valid, 32));
        void* p_d;
        if ((rc = grow_copy(ctx, F_DESC, sizeof(float) * DESC_LEN * (size_t)(done + chunk),
                            sizeof(float) * DESC_LEN * (size_t)done, &p_d)))
            return rc;
        p_desc = p_d;
        hook.begin("sift_desc");
        desc_kernel<<<(unsigned)((chunk + WARPS - 1) / WARPS), 32 * WARPS, 0, st>>>(
            kp, done, (int)chunk, (const int32_t*)p_pkp, (const double*)p_pth, table, (float*)p_desc,
            (uint8_t*)p_valid);
        SCK(cudaGetLastError());
        hook.end("sift_desc");
        done += chunk;
        size_t tb = 0;
        SCK(cub::DeviceSelect::Flagged(nullptr, tb, it, (const uint8_t*)p_valid, (uint32_t*)p_osel,
                                       (int*)p_nsel + 1, (int)done, st));
        SCK(A.get(F_TEMP, tb, &p_temp));
        SCK(cub::DeviceSelect::Flagged(p_temp, tb, it, (const uint8_t*)p_valid, (uint32_t*)p_osel,
                                       (int*)p_nsel + 1, (int)done, st));
        int nv = 0;
        SCK(cudaMemcpyAsync(&nv, (int*)p_nsel + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        SCK(cudaStreamSynchronize(st));
        n_valid = nv;
    }

    // sift.rs:543-544: the first max_features
    const int64_t n_out = std::min<int64_t>(n_valid, cap);
    out->width = w;
    out->height = h;
    out->n_raw = n_raw;
    out->n = (uint64_t)n_out;
    out->pts = (double*)std::malloc(sizeof(double) * 2 * std::max<int64_t>(n_out, 1));
    out->desc = (float*)std::malloc(sizeof(float) * DESC_LEN * std::max<int64_t>(n_out, 1));
    out->colors = (uint8_t*)std::malloc(3 * std::max<int64_t>(n_out, 1));
    if (!out->pts || !out->desc || !out->colors) {
        rcmvs_sift_frame_free(out);
        return sfail(ctx, RCMVS_E_NOMEM, "sift: host allocation failed");
    }
    if (n_out == 0) return RCMVS_OK;
    void *p_pts, *p_fdesc, *p_col;
    SCK(A.get(F_PTS, sizeof(double) * 2 * n_out, &p_pts));
    SCK(A.get(F_FDESC, sizeof(float) * DESC_LEN * n_out, &p_fdesc));
    SCK(A.get(F_COL, 3 * (size_t)n_out, &p_col));
    final_kernel<<<(int)((n_out + WARPS - 1) / WARPS), 32 * WARPS, 0, st>>>(
        (const uint32_t*)p_osel, (int)n_out, (const int32_t*)p_pkp, kp, table,
        (const float*)p_desc, (const uint8_t*)p_rgb, w, h, (double*)p_pts, (float*)p_fdesc, (uint8_t*)p_col);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(out->pts, p_pts, sizeof(double) * 2 * n_out, cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(out->desc, p_fdesc, sizeof(float) * DESC_LEN * n_out, cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(out->colors, p_col, 3 * (size_t)n_out, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    return RCMVS_OK;
}

}  // extern "C"
