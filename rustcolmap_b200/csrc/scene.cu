// scene.cu — seeded synthetic scene renderer (input generator for tests and
// benchmarks; not part of the stereo/fusion path).  Ray casting of rectangles,
// boxes and spheres with 4-octave value-noise texture.  Host and device run
// the same __host__ __device__ code; the build uses --fmad=false (device) and
// -ffp-contract=off (host), so both produce identical images.  Compiled as
// plain C++ (no __CUDACC__) it is the host renderer alone, for programs that
// must not load the CUDA library (device >= 0 is then refused).
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rcscene.h"

#ifdef __CUDACC__
#define HD __host__ __device__ __forceinline__
#else
#define HD inline
#endif

namespace {

thread_local std::string g_err;

struct RCam {
    int w, h;
    float f, cx, cy;
    float R[9];  // world->camera
    float C[3];  // centre in world
};

HD uint32_t mix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}

HD float lattice(int x, int y, int z, int seed) {
    uint32_t h = ((uint32_t)x * 0x8da6b343u) ^ ((uint32_t)y * 0xd8163841u) ^
                 ((uint32_t)z * 0xcb1ab31fu) ^ ((uint32_t)seed * 0x165667b1u);
    return (float)(mix32(h) >> 8) * (1.0f / 16777216.0f);
}

HD float smooth01(float t) { return t * t * (3.0f - 2.0f * t); }
HD float lerpf(float a, float b, float t) { return a + (b - a) * t; }

HD float vnoise(float x, float y, float z, int seed) {
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    float tx = smooth01(x - fx), ty = smooth01(y - fy), tz = smooth01(z - fz);
    float c000 = lattice(ix, iy, iz, seed), c100 = lattice(ix + 1, iy, iz, seed);
    float c010 = lattice(ix, iy + 1, iz, seed), c110 = lattice(ix + 1, iy + 1, iz, seed);
    float c001 = lattice(ix, iy, iz + 1, seed), c101 = lattice(ix + 1, iy, iz + 1, seed);
    float c011 = lattice(ix, iy + 1, iz + 1, seed), c111 = lattice(ix + 1, iy + 1, iz + 1, seed);
    float x00 = lerpf(c000, c100, tx), x10 = lerpf(c010, c110, tx);
    float x01 = lerpf(c001, c101, tx), x11 = lerpf(c011, c111, tx);
    return lerpf(lerpf(x00, x10, ty), lerpf(x01, x11, ty), tz);
}

// 4-octave fractal value noise in [0, 1].
HD float fbm4(float x, float y, float z, float freq, int seed) {
    float s = 0.f, a = 0.5f, norm = 0.f, fr = freq;
    for (int o = 0; o < 4; ++o) {
        s = s + a * vnoise(x * fr, y * fr, z * fr, seed + 1013 * o);
        norm = norm + a;
        a = a * 0.5f;
        fr = fr * 2.0f;
    }
    return s / norm;
}

HD float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

struct Hit {
    float s;
    float n[3];
    int prim;
    float a, b;  // rect-local coordinates
};

HD bool hit_rect(const rcscene_prim& p, const float* o, const float* d, Hit& h) {
    const float* P0 = p.p;
    const float* u = p.p + 3;
    const float* v = p.p + 6;
    float n[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    float denom = dot3(n, d);
    if (fabsf(denom) < 1e-12f) return false;
    float rel0[3] = {P0[0] - o[0], P0[1] - o[1], P0[2] - o[2]};
    float s = dot3(n, rel0) / denom;
    if (!(s > 1e-4f)) return false;
    float rel[3] = {o[0] + s * d[0] - P0[0], o[1] + s * d[1] - P0[1], o[2] + s * d[2] - P0[2]};
    float a = dot3(rel, u), b = dot3(rel, v);
    if (!(a >= 0.f && a <= p.p[9] && b >= 0.f && b <= p.p[10])) return false;
    h.s = s;
    float sg = denom < 0.f ? 1.0f : -1.0f;
    h.n[0] = sg * n[0];
    h.n[1] = sg * n[1];
    h.n[2] = sg * n[2];
    h.a = a;
    h.b = b;
    return true;
}

HD bool hit_box(const rcscene_prim& p, const float* o, const float* d, Hit& h) {
    float tn = -INFINITY, tf = INFINITY;
    int axn = 0, axf = 0;
    for (int a = 0; a < 3; ++a) {
        float lo = p.p[a], hi = p.p[3 + a];
        if (d[a] == 0.f) {
            if (o[a] < lo || o[a] > hi) return false;
            continue;
        }
        float t1 = (lo - o[a]) / d[a], t2 = (hi - o[a]) / d[a];
        if (t1 > t2) {
            float tmp = t1;
            t1 = t2;
            t2 = tmp;
        }
        if (t1 > tn) {
            tn = t1;
            axn = a;
        }
        if (t2 < tf) {
            tf = t2;
            axf = a;
        }
    }
    if (tn > tf || tf < 1e-4f) return false;
    int ax = axn;
    float s = tn;
    float sg = d[ax] > 0.f ? -1.0f : 1.0f;
    if (!(tn > 1e-4f)) {  // origin inside the box: exit face
        s = tf;
        ax = axf;
        sg = d[ax] > 0.f ? -1.0f : 1.0f;
    }
    h.s = s;
    h.n[0] = h.n[1] = h.n[2] = 0.f;
    h.n[ax] = sg;
    return true;
}

HD bool hit_sphere(const rcscene_prim& p, const float* o, const float* d, Hit& h) {
    float oc[3] = {o[0] - p.p[0], o[1] - p.p[1], o[2] - p.p[2]};
    float A = dot3(d, d), B = dot3(oc, d), Cc = dot3(oc, oc) - p.p[3] * p.p[3];
    float disc = B * B - A * Cc;
    if (disc < 0.f) return false;
    float sq = sqrtf(disc);
    float s = (-B - sq) / A;
    if (!(s > 1e-4f)) s = (-B + sq) / A;
    if (!(s > 1e-4f)) return false;
    h.s = s;
    float P[3] = {o[0] + s * d[0] - p.p[0], o[1] + s * d[1] - p.p[1], o[2] + s * d[2] - p.p[2]};
    float inv = 1.0f / p.p[3];
    h.n[0] = P[0] * inv;
    h.n[1] = P[1] * inv;
    h.n[2] = P[2] * inv;
    return true;
}

HD bool trace(const rcscene_prim* prims, int np, const float* o, const float* d, Hit& best) {
    best.s = INFINITY;
    best.prim = -1;
    for (int i = 0; i < np; ++i) {
        Hit h;
        bool ok = false;
        if (prims[i].kind == RCSCENE_RECT)
            ok = hit_rect(prims[i], o, d, h);
        else if (prims[i].kind == RCSCENE_BOX)
            ok = hit_box(prims[i], o, d, h);
        else
            ok = hit_sphere(prims[i], o, d, h);
        if (ok && h.s < best.s) {
            best = h;
            best.prim = i;
        }
    }
    return best.prim >= 0;
}

HD float shade(const rcscene_prim* prims, const rcscene_patch* patches, int npatch, const float* o,
               const float* d, const Hit& h) {
    const rcscene_prim& p = prims[h.prim];
    if (p.kind == RCSCENE_RECT) {
        float val = -1.f;
        for (int q = 0; q < npatch; ++q) {
            const rcscene_patch& r = patches[q];
            if (r.prim == h.prim && h.a >= r.u0 && h.a <= r.u1 && h.b >= r.v0 && h.b <= r.v1) val = r.value;
        }
        if (val >= 0.f) return val;
    }
    float P[3] = {o[0] + h.s * d[0], o[1] + h.s * d[1], o[2] + h.s * d[2]};
    float n = fbm4(P[0], P[1], P[2], p.tex_freq, p.tex_seed);
    float t = (n - 0.5f) * 2.2f + 0.5f;
    t = t < 0.f ? 0.f : (t > 1.f ? 1.f : t);
    return p.tex_lo + (p.tex_hi - p.tex_lo) * t;
}

HD void render_px(const rcscene_prim* prims, int np, const rcscene_patch* patches, int npatch,
                  const RCam& c, int x, int y, int ss, uint8_t* gray, float* depth, float* normal) {
    size_t i = (size_t)y * c.w + x;
    float acc = 0.f;
    for (int sy = 0; sy < ss; ++sy)
        for (int sx = 0; sx < ss; ++sx) {
            float ox = ((float)sx + 0.5f) / (float)ss - 0.5f;
            float oy = ((float)sy + 0.5f) / (float)ss - 0.5f;
            float dc[3] = {((float)x + ox - c.cx) / c.f, ((float)y + oy - c.cy) / c.f, 1.0f};
            float dw[3] = {c.R[0] * dc[0] + c.R[3] * dc[1] + c.R[6] * dc[2],
                           c.R[1] * dc[0] + c.R[4] * dc[1] + c.R[7] * dc[2],
                           c.R[2] * dc[0] + c.R[5] * dc[1] + c.R[8] * dc[2]};
            Hit h;
            if (trace(prims, np, c.C, dw, h)) acc = acc + shade(prims, patches, npatch, c.C, dw, h);
        }
    float g = acc / (float)(ss * ss);
    int gi = (int)(g + 0.5f);
    gray[i] = (uint8_t)(gi < 0 ? 0 : (gi > 255 ? 255 : gi));
    // ground truth from the pixel-centre ray
    float dc[3] = {((float)x - c.cx) / c.f, ((float)y - c.cy) / c.f, 1.0f};
    float dw[3] = {c.R[0] * dc[0] + c.R[3] * dc[1] + c.R[6] * dc[2],
                   c.R[1] * dc[0] + c.R[4] * dc[1] + c.R[7] * dc[2],
                   c.R[2] * dc[0] + c.R[5] * dc[1] + c.R[8] * dc[2]};
    Hit h;
    bool ok = trace(prims, np, c.C, dw, h);
    depth[i] = ok ? h.s : 0.f;
    if (normal) {
        for (int a = 0; a < 3; ++a)
            normal[3 * i + a] = ok ? c.R[3 * a] * h.n[0] + c.R[3 * a + 1] * h.n[1] + c.R[3 * a + 2] * h.n[2] : 0.f;
    }
}

#ifdef __CUDACC__
__global__ void render_kernel(const rcscene_prim* prims, int np, const rcscene_patch* patches, int npatch,
                              RCam c, int ss, uint8_t* gray, float* depth, float* normal) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= c.w || y >= c.h) return;
    render_px(prims, np, patches, npatch, c, x, y, ss, gray, depth, normal);
}

#endif

RCam make_cam(const rcscene_cam& k) {
    RCam c;
    c.w = k.w;
    c.h = k.h;
    c.f = (float)k.f;
    c.cx = (float)k.cx;
    c.cy = (float)k.cy;
    for (int i = 0; i < 9; ++i) c.R[i] = (float)k.R[i];
    for (int a = 0; a < 3; ++a)  // C = -R^T t, in f64 then cast
        c.C[a] = (float)(-(k.R[a] * k.t[0] + k.R[3 + a] * k.t[1] + k.R[6 + a] * k.t[2]));
    return c;
}

#ifdef __CUDACC__
#define CK(x)                                                                  \
    do {                                                                       \
        cudaError_t e_ = (x);                                                  \
        if (e_ != cudaSuccess) {                                               \
            g_err = std::string(#x) + ": " + cudaGetErrorString(e_);           \
            rc = -2;                                                           \
            goto done;                                                         \
        }                                                                      \
    } while (0)
#endif

}  // namespace

extern "C" const char* rcscene_last_error(void) { return g_err.c_str(); }

extern "C" int rcscene_render(const rcscene_prim* prims, int32_t n_prims, const rcscene_patch* patches,
                              int32_t n_patches, const rcscene_cam* cams, int32_t n_cams,
                              int32_t supersample, int32_t device, uint8_t* const* gray_out,
                              float* const* depth_out, float* const* normal_out) {
    if (!prims || n_prims <= 0 || (n_patches > 0 && !patches) || !cams || n_cams <= 0 || !gray_out ||
        !depth_out || supersample < 1) {
        g_err = "rcscene_render: bad argument";
        return -1;
    }
    for (int v = 0; v < n_cams; ++v)
        if (cams[v].w <= 0 || cams[v].h <= 0 || !gray_out[v] || !depth_out[v]) {
            g_err = "rcscene_render: bad camera or output";
            return -1;
        }
    if (device < 0) {
        for (int v = 0; v < n_cams; ++v) {
            RCam c = make_cam(cams[v]);
            float* nrm = normal_out ? normal_out[v] : nullptr;
            unsigned nt = std::thread::hardware_concurrency();
            if (nt < 1) nt = 1;
            std::atomic<int> next(0);
            std::vector<std::thread> ts;
            for (unsigned t = 0; t < nt; ++t)
                ts.emplace_back([&] {
                    for (;;) {
                        int y = next.fetch_add(1);
                        if (y >= c.h) break;
                        for (int x = 0; x < c.w; ++x)
                            render_px(prims, n_prims, patches, n_patches, c, x, y, supersample, gray_out[v],
                                      depth_out[v], nrm);
                    }
                });
            for (auto& t : ts) t.join();
        }
        return 0;
    }
#ifndef __CUDACC__
    g_err = "rcscene_render: the host-only library renders on the host only (device = -1)";
    return -1;
#else
    int rc = 0;
    rcscene_prim* dprims = nullptr;
    rcscene_patch* dpatch = nullptr;
    uint8_t* dg = nullptr;
    float *dd = nullptr, *dn = nullptr;
    size_t maxpx = 0;
    for (int v = 0; v < n_cams; ++v) maxpx = std::max(maxpx, (size_t)cams[v].w * cams[v].h);
    CK(cudaSetDevice(device));
    CK(cudaMalloc(&dprims, sizeof(rcscene_prim) * n_prims));
    CK(cudaMemcpy(dprims, prims, sizeof(rcscene_prim) * n_prims, cudaMemcpyHostToDevice));
    if (n_patches > 0) {
        CK(cudaMalloc(&dpatch, sizeof(rcscene_patch) * n_patches));
        CK(cudaMemcpy(dpatch, patches, sizeof(rcscene_patch) * n_patches, cudaMemcpyHostToDevice));
    }
    CK(cudaMalloc(&dg, maxpx));
    CK(cudaMalloc(&dd, maxpx * sizeof(float)));
    if (normal_out) CK(cudaMalloc(&dn, maxpx * 3 * sizeof(float)));
    for (int v = 0; v < n_cams; ++v) {
        RCam c = make_cam(cams[v]);
        dim3 blk(32, 8), grd((c.w + 31) / 32, (c.h + 7) / 8);
        render_kernel<<<grd, blk>>>(dprims, n_prims, dpatch, n_patches, c, supersample, dg, dd,
                                    normal_out ? dn : nullptr);
        CK(cudaGetLastError());
        size_t npx = (size_t)c.w * c.h;
        CK(cudaMemcpy(gray_out[v], dg, npx, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(depth_out[v], dd, npx * sizeof(float), cudaMemcpyDeviceToHost));
        if (normal_out && normal_out[v]) CK(cudaMemcpy(normal_out[v], dn, npx * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    }
done:
    cudaFree(dprims);
    cudaFree(dpatch);
    cudaFree(dg);
    cudaFree(dd);
    cudaFree(dn);
    return rc;
#endif
}
