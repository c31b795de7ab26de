// depthvis.cu — depth-map visualisation on sm_100a.
//
// Restates mvs/src/fuse.rs:241-268 (save_depth_vis): the 2nd and 98th
// percentiles of a map's valid depths (z > 0) set the grey scale; pixel value
// 0 for invalid depth, else (255 * (1 - clamp((z - lo) / range, 0, 1))) as u8
// in f32 (near = bright).
//
//   select  valid depths, compacted (CUB select)
//   sort    their bit patterns (positive floats order as unsigned integers;
//           CUB radix sort), then the two order statistics the reference
//           indexes: ds[(n * 0.02) as usize] and ds[(n * 0.98) as usize - 1]
//           (n >= 32; else lo = 0, hi = 1)
//   map     one thread per pixel
//
// The PNG file is written on the host with zlib (rcmvs_write_png_gray): an
// 8-bit grey PNG whose decoded pixels are the image; the reference's `image`
// crate encoder compresses differently, so files differ in bytes, not pixels.
#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "ctx_internal.cuh"

namespace rcmvs {

namespace {

struct ValidDepth {
    __host__ __device__ bool operator()(const float z) const { return z > 0.0f; }
};

// Rust `f32 as u8`: truncation toward zero, saturating to [0, 255], NaN -> 0.
__device__ __forceinline__ uint8_t f32_to_u8(float v) {
    if (!(v > 0.0f)) return 0;
    if (v >= 255.0f) return 255;
    return (uint8_t)(int)v;
}

// fuse.rs:251-258
__global__ void vis_kernel(const float* __restrict__ depth, int64_t n, float lo, float range,
                           uint8_t* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float z = depth[i];
    uint8_t val = 0;
    if (!(z <= 0.0f)) {
        float t = (z - lo) / range;
        // f32::clamp(0.0, 1.0): NaN stays NaN
        if (t < 0.0f) t = 0.0f;
        else if (t > 1.0f) t = 1.0f;
        val = f32_to_u8(255.0f * (1.0f - t));
    }
    out[i] = val;
}

int vfail(rcmvs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

#define VCK(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            return vfail(ctx, e_ == cudaErrorMemoryAllocation ? RCMVS_E_NOMEM : RCMVS_E_CUDA,    \
                         std::string(#x) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

// Arena slots (of the arena passed in): 50-54.
enum { V_VALID = 50, V_SORTED = 51, V_NSEL = 52, V_TEMP = 53, V_OUT = 54 };

// Visualises n device depths into d_out (device, n bytes); lohi gets the
// (lo, hi) percentiles.  Synchronises once to size the selection.
int depth_vis_device(rcmvs_ctx* ctx, DeviceArena& A, const float* d_depth, int64_t n, uint8_t* d_out, float lohi[2]) {
    if (n <= 0 || n > INT32_MAX) return vfail(ctx, RCMVS_E_LIMIT, "depth map size out of range");
    cudaStream_t st = ctx->stream;
    void *p_valid, *p_sorted, *p_nsel, *p_temp;
    VCK(A.get(V_VALID, sizeof(float) * n, &p_valid));
    VCK(A.get(V_SORTED, sizeof(uint32_t) * n, &p_sorted));
    VCK(A.get(V_NSEL, sizeof(int), &p_nsel));
    size_t t_sel = 0, t_sort = 0;
    VCK(cub::DeviceSelect::If(nullptr, t_sel, d_depth, (float*)p_valid, (int*)p_nsel, (int)n, ValidDepth(), st));
    VCK(cub::DeviceRadixSort::SortKeys(nullptr, t_sort, (const uint32_t*)p_valid, (uint32_t*)p_sorted, (int)n, 0, 32,
                                       st));
    VCK(A.get(V_TEMP, std::max(t_sel, t_sort), &p_temp));
    VCK(cub::DeviceSelect::If(p_temp, t_sel, d_depth, (float*)p_valid, (int*)p_nsel, (int)n, ValidDepth(), st));
    int nsel = 0;
    VCK(cudaMemcpyAsync(&nsel, p_nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
    VCK(cudaStreamSynchronize(st));
    float lo = 0.0f, hi = 1.0f;  // fuse.rs:245-249
    if (nsel >= 32) {
        VCK(cub::DeviceRadixSort::SortKeys(p_temp, t_sort, (const uint32_t*)p_valid, (uint32_t*)p_sorted, nsel, 0, 32,
                                           st));
        const size_t i_lo = (size_t)((double)nsel * 0.02);
        const size_t i_hi = (size_t)((double)nsel * 0.98) - 1;
        VCK(cudaMemcpyAsync(&lo, (const uint32_t*)p_sorted + i_lo, 4, cudaMemcpyDeviceToHost, st));
        VCK(cudaMemcpyAsync(&hi, (const uint32_t*)p_sorted + i_hi, 4, cudaMemcpyDeviceToHost, st));
        VCK(cudaStreamSynchronize(st));
    }
    const float range = std::fmax(hi - lo, 1e-9f);  // fuse.rs:250
    vis_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_depth, n, lo, range, d_out);
    VCK(cudaGetLastError());
    if (lohi) {
        lohi[0] = lo;
        lohi[1] = hi;
    }
    return RCMVS_OK;
}

void put_be32(std::vector<unsigned char>& b, uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
}

void put_chunk(std::vector<unsigned char>& b, const char* type, const unsigned char* data, size_t len) {
    put_be32(b, (uint32_t)len);
    const size_t start = b.size();
    b.insert(b.end(), type, type + 4);
    if (len) b.insert(b.end(), data, data + len);
    const uLong crc = crc32(0L, b.data() + start, (uInt)(4 + len));
    put_be32(b, (uint32_t)crc);
}

}  // namespace
}  // namespace rcmvs

using namespace rcmvs;

extern "C" {

int rcmvs_depth_vis(rcmvs_ctx* ctx, const float* depth, int32_t w, int32_t h, uint8_t* out, float* lo_hi) {
    if (!ctx || !depth || !out || w <= 0 || h <= 0) return vfail(ctx, RCMVS_E_ARG, "rcmvs_depth_vis: bad argument");
    VCK(cudaSetDevice(ctx->device));
    const int64_t n = (int64_t)w * h;
    void *p_in, *p_out;
    VCK(ctx->arena.get(55, sizeof(float) * n, &p_in));
    VCK(ctx->arena.get(V_OUT, n, &p_out));
    VCK(cudaMemcpyAsync(p_in, depth, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
    float lh[2];
    int rc = depth_vis_device(ctx, ctx->arena, (const float*)p_in, n, (uint8_t*)p_out, lh);
    if (rc) return rc;
    VCK(cudaMemcpyAsync(out, p_out, n, cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaStreamSynchronize(ctx->stream));
    if (lo_hi) {
        lo_hi[0] = lh[0];
        lo_hi[1] = lh[1];
    }
    return RCMVS_OK;
}

int rcmvs_scene_depth_vis(rcmvs_ctx* ctx, rcmvs_scene* sc, int32_t view, uint8_t* out, float* lo_hi) {
    if (!ctx || !sc || !out || view < 0 || view >= sc->n_views)
        return vfail(ctx, RCMVS_E_ARG, "rcmvs_scene_depth_vis: bad argument");
    if (!sc->has_depth[view]) return vfail(ctx, RCMVS_E_STATE, "view has no depth map");
    VCK(cudaSetDevice(ctx->device));
    const DevView& V = sc->views[view];
    const int64_t n = (int64_t)V.w * V.h;
    void* p_out;
    VCK(sc->arena.get(V_OUT, n, &p_out));
    float lh[2];
    int rc = depth_vis_device(ctx, sc->arena, sc->depth + V.off, n, (uint8_t*)p_out, lh);
    if (rc) return rc;
    VCK(cudaMemcpyAsync(out, p_out, n, cudaMemcpyDeviceToHost, ctx->stream));
    VCK(cudaStreamSynchronize(ctx->stream));
    if (lo_hi) {
        lo_hi[0] = lh[0];
        lo_hi[1] = lh[1];
    }
    return RCMVS_OK;
}

int rcmvs_write_png_gray(const char* path, const uint8_t* img, int32_t w, int32_t h) {
    if (!path || !img || w <= 0 || h <= 0) return RCMVS_E_ARG;
    // raw scanlines, each prefixed by filter type 0
    std::vector<unsigned char> raw((size_t)(w + 1) * h);
    for (int32_t y = 0; y < h; ++y) {
        raw[(size_t)y * (w + 1)] = 0;
        std::memcpy(&raw[(size_t)y * (w + 1) + 1], img + (size_t)y * w, (size_t)w);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<unsigned char> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) return RCMVS_E_NOMEM;
    std::vector<unsigned char> b = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    unsigned char ihdr[13];
    for (int i = 0; i < 4; ++i) {
        ihdr[i] = (unsigned char)((uint32_t)w >> (24 - 8 * i));
        ihdr[4 + i] = (unsigned char)((uint32_t)h >> (24 - 8 * i));
    }
    ihdr[8] = 8;   // bit depth
    ihdr[9] = 0;   // grey
    ihdr[10] = 0;  // deflate
    ihdr[11] = 0;  // adaptive filtering (type 0 used)
    ihdr[12] = 0;  // no interlace
    put_chunk(b, "IHDR", ihdr, 13);
    put_chunk(b, "IDAT", z.data(), zlen);
    put_chunk(b, "IEND", nullptr, 0);
    FILE* f = std::fopen(path, "wb");
    if (!f) return RCMVS_E_IO;
    const bool ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
    return (std::fclose(f) == 0 && ok) ? RCMVS_OK : RCMVS_E_IO;
}

}  // extern "C"
