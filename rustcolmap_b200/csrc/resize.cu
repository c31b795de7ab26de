// resize.cu — images at the stereo working resolution, on sm_100a.
//
// Restates the image preparation of mvs::load_views (mvs/src/lib.rs:183-194):
// `DynamicImage::resize_exact(mw, mh, FilterType::Triangle)` when the size
// changes, then `to_luma8` and `to_rgb8`.  The resize is the `image` crate's
// (0.24, Cargo.lock; not part of the reference tree) separable resampler,
// imageops::resize: a vertical pass from the 8-bit image into an f32 image of
// mh rows, then a horizontal pass into mw columns rounded back to u8.  Along
// an axis of n input samples resampled to m, output sample o reads
//
//   ratio  = n / m (f32),  s = max(ratio, 1),  support = 1 * s
//   centre = (o + 0.5) * ratio
//   taps   [left, right): left  = clamp(floor(centre - support), 0, n - 1)
//                         right = clamp(ceil(centre + support), left + 1, n)
//   weight of tap i: tri((i - (centre - 0.5)) / s), tri(x) = |x| < 1 ? 1 - |x| : 0,
//                    each divided by the f32 sum of all of them (summed in i order)
//   value = sum over i (in order) of sample[i] * weight[i], in f32
//
// and the horizontal pass stores round(clamp(value, 0, 255)) (round half away
// from zero).  Channels resample independently; alpha is dropped.  Luma of
// RGB is (2126 R + 7152 G + 722 B) / 10000 in integers.  The library builds
// with --fmad=false, so every product and sum rounds as the f32 operations
// written above.
//
//   taps_kernel    one thread per output coordinate of an axis: its first
//                  tap, tap count and normalised weights (a table of m rows)
//   vert_kernel    one thread per (output row, input column, channel): the
//                  f32 image of mh rows; a warp reads consecutive bytes of
//                  one input row per tap and shares its weight row
//   horiz_kernel   one thread per output pixel: its channels, rounded, with
//                  grey and RGB written together
//   convert_kernel no resize: to_luma8 / to_rgb8 of the input
//
// All of it is HBM-bound byte and f32 work, small beside stereo: a 4000x3000
// RGB image brought to 1920x1440 reads 36 MB, writes and reads a 69 MB f32
// intermediate and writes 11 MB.
#include <cmath>
#include <cstring>
#include <string>

#include "ctx_internal.cuh"

namespace rcmvs {

namespace {

constexpr int kMaxSide = 1 << 23;

__device__ __forceinline__ uint8_t luma709(uint32_t r, uint32_t g, uint32_t b) {
    return (uint8_t)((2126u * r + 7152u * g + 722u * b) / 10000u);
}

// An upper bound on right - left for every output coordinate (host and
// device compute s the same way): ceil(c + s) - floor(c - s) < 2s + 2 plus
// the rounding of c +- s, so 2s + 3 taps always suffice.
int taps_bound(int n, int m) {
    const float ratio = (float)n / (float)m;
    const float s = ratio < 1.0f ? 1.0f : ratio;
    const long long b = (long long)std::ceil(2.0 * (double)s) + 3;
    return (int)(b < (long long)n ? b : (long long)n);
}

__global__ void taps_kernel(int32_t n, int32_t m, int32_t maxt, int32_t* __restrict__ first,
                            int32_t* __restrict__ count, float* __restrict__ weight, int* __restrict__ err) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= m) return;
    const float ratio = __fdiv_rn((float)n, (float)m);
    const float s = ratio < 1.0f ? 1.0f : ratio;
    const float support = __fmul_rn(1.0f, s);
    float c = __fmul_rn(__fadd_rn((float)o, 0.5f), ratio);
    long long l = (long long)floorf(__fsub_rn(c, support));
    l = l < 0 ? 0 : (l > n - 1 ? n - 1 : l);
    long long r = (long long)ceilf(__fadd_rn(c, support));
    r = r < l + 1 ? l + 1 : (r > n ? n : r);
    c = __fsub_rn(c, 0.5f);
    int cnt = (int)(r - l);
    if (cnt > maxt) {  // never taken: maxt bounds every count
        atomicExch(err, 1);
        cnt = maxt;
    }
    float* w = weight + (size_t)o * maxt;
    float sum = 0.0f;
    for (int i = 0; i < cnt; ++i) {
        const float x = __fdiv_rn(__fsub_rn((float)(l + i), c), s);
        const float ax = fabsf(x);
        const float wi = ax < 1.0f ? __fsub_rn(1.0f, ax) : 0.0f;
        w[i] = wi;
        sum = __fadd_rn(sum, wi);
    }
    for (int i = 0; i < cnt; ++i) w[i] = __fdiv_rn(w[i], sum);
    first[o] = (int32_t)l;
    count[o] = cnt;
}

// tmp[(y * w + x) * nc + c] for output row y, input column x, channel c < nc
// of an input with `channels` bytes per pixel.
__global__ void vert_kernel(const uint8_t* __restrict__ img, int32_t w, int32_t channels, int32_t nc, int32_t mh,
                            const int32_t* __restrict__ first, const int32_t* __restrict__ count,
                            const float* __restrict__ weight, int32_t maxt, float* __restrict__ tmp) {
    const int64_t row = (int64_t)w * nc;
    const int64_t total = row * mh;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / row);
        const int64_t j = i - (int64_t)y * row;
        const int x = (int)(j / nc), c = (int)(j - (int64_t)x * nc);
        const int l = first[y], cnt = count[y];
        const float* wy = weight + (size_t)y * maxt;
        const uint8_t* src = img + ((int64_t)l * w + x) * channels + c;
        const int64_t step = (int64_t)w * channels;
        float t = 0.0f;
        for (int k = 0; k < cnt; ++k) t = __fadd_rn(t, __fmul_rn((float)src[k * step], wy[k]));
        tmp[i] = t;
    }
}

__device__ __forceinline__ uint8_t to_u8(float t) {
    t = t < 0.0f ? 0.0f : (t > 255.0f ? 255.0f : t);
    return (uint8_t)(int)roundf(t);
}

template <int NC>
__global__ void horiz_kernel(const float* __restrict__ tmp, int32_t w, int32_t mw, int32_t mh,
                             const int32_t* __restrict__ first, const int32_t* __restrict__ count,
                             const float* __restrict__ weight, int32_t maxt, uint8_t* __restrict__ gray,
                             uint8_t* __restrict__ rgb) {
    const int64_t total = (int64_t)mw * mh;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / mw), x = (int)(i - (int64_t)y * mw);
        const int l = first[x], cnt = count[x];
        const float* wx = weight + (size_t)x * maxt;
        const float* src = tmp + ((int64_t)y * w + l) * NC;
        uint8_t v[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            float t = 0.0f;
            for (int k = 0; k < cnt; ++k) t = __fadd_rn(t, __fmul_rn(src[k * NC + c], wx[k]));
            v[c] = to_u8(t);
        }
        if constexpr (NC == 1) {
            gray[i] = v[0];
            rgb[3 * i] = rgb[3 * i + 1] = rgb[3 * i + 2] = v[0];
        } else {
            gray[i] = luma709(v[0], v[1], v[2]);
            rgb[3 * i] = v[0];
            rgb[3 * i + 1] = v[1];
            rgb[3 * i + 2] = v[2];
        }
    }
}

__global__ void convert_kernel(const uint8_t* __restrict__ img, int64_t n, int32_t channels,
                               uint8_t* __restrict__ gray, uint8_t* __restrict__ rgb) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t* p = img + i * channels;
        if (channels < 3) {
            gray[i] = p[0];
            rgb[3 * i] = rgb[3 * i + 1] = rgb[3 * i + 2] = p[0];
        } else {
            gray[i] = luma709(p[0], p[1], p[2]);
            rgb[3 * i] = p[0];
            rgb[3 * i + 1] = p[1];
            rgb[3 * i + 2] = p[2];
        }
    }
}

int rfail(rcmvs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

#define RCK(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return rfail(ctx, e_ == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,    \
                         std::string(#x) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

// Context arena slots 60-68.
enum { R_IN = 60, R_TMP = 61, R_GRAY = 62, R_RGB = 63, R_VIDX = 64, R_VW = 65, R_HIDX = 66, R_HW = 67, R_ERR = 68 };

unsigned grid_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace

int resize_check(rcmvs_ctx* ctx, int w, int h, int channels, int mw, int mh) {
    if (w <= 0 || h <= 0 || mw <= 0 || mh <= 0 || channels < 1 || channels > 4)
        return rfail(ctx, RCMVS_E_ARG, "resize: bad size or channel count");
    if (w > kMaxSide || h > kMaxSide || mw > kMaxSide || mh > kMaxSide || (int64_t)w * h > INT32_MAX ||
        (int64_t)mw * mh > INT32_MAX || (int64_t)w * mh > INT32_MAX)
        return rfail(ctx, RCMVS_E_LIMIT, "resize: image side above 2^23 or more than 2^31 pixels");
    return RCMVS_OK;
}

int resize_device(rcmvs_ctx* ctx, const uint8_t* d_in, int w, int h, int channels, int mw, int mh, uint8_t* d_gray,
                  uint8_t* d_rgb, const int** d_err) {
    cudaStream_t st = ctx->stream;
    DeviceArena& A = ctx->arena;
    const int64_t n_in = (int64_t)w * h, n_out = (int64_t)mw * mh;
    *d_err = nullptr;
    if (mw == w && mh == h) {  // mvs/src/lib.rs:188-192: no resize
        convert_kernel<<<grid_for(n_in), 256, 0, st>>>(d_in, n_in, channels, d_gray, d_rgb);
        RCK(cudaGetLastError());
        return RCMVS_OK;
    }
    const int nc = channels < 3 ? 1 : 3;
    const int tv = taps_bound(h, mh), th = taps_bound(w, mw);
    void *p_tmp, *p_vidx, *p_vw, *p_hidx, *p_hw, *p_err;
    RCK(A.get(R_TMP, sizeof(float) * (size_t)w * mh * nc, &p_tmp));
    RCK(A.get(R_VIDX, sizeof(int32_t) * 2 * (size_t)mh, &p_vidx));
    RCK(A.get(R_VW, sizeof(float) * (size_t)mh * tv, &p_vw));
    RCK(A.get(R_HIDX, sizeof(int32_t) * 2 * (size_t)mw, &p_hidx));
    RCK(A.get(R_HW, sizeof(float) * (size_t)mw * th, &p_hw));
    RCK(A.get(R_ERR, sizeof(int), &p_err));
    RCK(cudaMemsetAsync(p_err, 0, sizeof(int), st));
    int32_t* vfirst = (int32_t*)p_vidx;
    int32_t* hfirst = (int32_t*)p_hidx;
    taps_kernel<<<(mh + 127) / 128, 128, 0, st>>>(h, mh, tv, vfirst, vfirst + mh, (float*)p_vw, (int*)p_err);
    RCK(cudaGetLastError());
    taps_kernel<<<(mw + 127) / 128, 128, 0, st>>>(w, mw, th, hfirst, hfirst + mw, (float*)p_hw, (int*)p_err);
    RCK(cudaGetLastError());
    vert_kernel<<<grid_for((int64_t)w * nc * mh), 256, 0, st>>>(d_in, w, channels, nc, mh, vfirst, vfirst + mh,
                                                                 (const float*)p_vw, tv, (float*)p_tmp);
    RCK(cudaGetLastError());
    if (nc == 1)
        horiz_kernel<1><<<grid_for(n_out), 256, 0, st>>>((const float*)p_tmp, w, mw, mh, hfirst, hfirst + mw,
                                                          (const float*)p_hw, th, d_gray, d_rgb);
    else
        horiz_kernel<3><<<grid_for(n_out), 256, 0, st>>>((const float*)p_tmp, w, mw, mh, hfirst, hfirst + mw,
                                                          (const float*)p_hw, th, d_gray, d_rgb);
    RCK(cudaGetLastError());
    *d_err = (const int*)p_err;
    return RCMVS_OK;
}

}  // namespace rcmvs

using namespace rcmvs;

extern "C" {

int rcmvs_working_size(int32_t w, int32_t h, uint32_t max_dim, int32_t* mw, int32_t* mh) {
    if (w <= 0 || h <= 0 || !mw || !mh) return RCMVS_E_ARG;
    // mvs/src/lib.rs:185-187: f64 scale, round half away from zero, `as u32`, at least 16
    const double s = std::fmin((double)max_dim / (double)(w > h ? w : h), 1.0);
    const double a = std::round((double)w * s), b = std::round((double)h * s);
    *mw = (int32_t)(a < 16.0 ? 16.0 : a);
    *mh = (int32_t)(b < 16.0 ? 16.0 : b);
    return RCMVS_OK;
}

int rcmvs_resize_view(rcmvs_ctx* ctx, const uint8_t* img, int32_t w, int32_t h, int32_t channels, int32_t mw,
                      int32_t mh, uint8_t* gray_out, uint8_t* rgb_out) {
    if (!ctx || !img) return rfail(ctx, RCMVS_E_ARG, "rcmvs_resize_view: bad argument");
    int rc = resize_check(ctx, w, h, channels, mw, mh);
    if (rc) return rc;
    RCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    DeviceArena& A = ctx->arena;
    const int64_t n_in = (int64_t)w * h, n_out = (int64_t)mw * mh;
    void *p_in, *p_gray, *p_rgb;
    RCK(A.get(R_IN, (size_t)n_in * channels, &p_in));
    RCK(A.get(R_GRAY, (size_t)n_out, &p_gray));
    RCK(A.get(R_RGB, (size_t)n_out * 3, &p_rgb));
    RCK(cudaMemcpyAsync(p_in, img, (size_t)n_in * channels, cudaMemcpyHostToDevice, st));
    const int* d_err = nullptr;
    rc = resize_device(ctx, (const uint8_t*)p_in, w, h, channels, mw, mh, (uint8_t*)p_gray, (uint8_t*)p_rgb, &d_err);
    if (rc) return rc;
    int bad = 0;
    if (d_err) RCK(cudaMemcpyAsync(&bad, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (gray_out) RCK(cudaMemcpyAsync(gray_out, p_gray, (size_t)n_out, cudaMemcpyDeviceToHost, st));
    if (rgb_out) RCK(cudaMemcpyAsync(rgb_out, p_rgb, (size_t)n_out * 3, cudaMemcpyDeviceToHost, st));
    RCK(cudaStreamSynchronize(st));
    if (bad) return rfail(ctx, RCMVS_E_CUDA, "rcmvs_resize_view: tap table overflow");
    return RCMVS_OK;
}

}  // extern "C"
