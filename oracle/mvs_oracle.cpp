// mvs_oracle.cpp — CPU oracle for the dense-MVS path (TEST INFRASTRUCTURE).
//
// A statement-by-statement restatement of the reference `mvs` crate, used only
// by tests, the smoke check and the CPU-baseline leg of bench.py as the
// checker.  It is never linked into the product library.
//
// Build: -O3 -ffp-contract=off, no fast-math (see oracle/Makefile).  Rust f32
// and f64 arithmetic is IEEE with no contraction, so the same expression tree
// evaluated here in the same order gives the same bits.
//
// PARITY UNPINNED: the reference (Rust) cannot be compiled where this was
// written and ships no golden vectors; see the header for what pins it.

#include "mvs_oracle.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <thread>
#include <tuple>
#include <vector>

namespace {

// Parallel loop over [0, n) — stands in for rayon's par_iter / par_chunks_mut.
// Every iteration writes disjoint outputs, so the schedule cannot change
// results.
template <class F>
void par_for(int64_t n, int nthreads, F&& f) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads < 1) nthreads = 1;
    if (nthreads == 1 || n <= 1) {
        for (int64_t i = 0; i < n; ++i) f(i, 0);
        return;
    }
    if (nthreads > n) nthreads = (int)n;
    std::atomic<int64_t> next(0);
    std::vector<std::thread> ts;
    for (int t = 0; t < nthreads; ++t) {
        ts.emplace_back([&, t] {
            for (;;) {
                int64_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i, t);
            }
        });
    }
    for (auto& t : ts) t.join();
}

inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Rust `f64 as i32`: truncate toward zero, saturate, NaN -> 0.
inline int32_t f64_to_i32(double v) {
    if (std::isnan(v)) return 0;
    if (v >= 2147483648.0) return INT32_MAX;
    if (v <= -2147483649.0) return INT32_MIN;
    return (int32_t)v;
}
// Rust `f64 as i64`.
inline int64_t f64_to_i64(double v) {
    if (std::isnan(v)) return 0;
    if (v >= 9223372036854775808.0) return INT64_MAX;
    if (v < -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}
// Rust `f64 as u8`.
inline uint8_t f64_to_u8(double v) {
    if (std::isnan(v) || v <= 0.0) return 0;
    if (v >= 255.0) return 255;
    return (uint8_t)v;
}

// nalgebra Matrix3 * Vector3 (gemv, k ascending: mvs uses 3x3 products only).
inline void mat3_vec(const double* m, const double* v, double* o) {
    for (int i = 0; i < 3; ++i) o[i] = m[3 * i + 0] * v[0] + m[3 * i + 1] * v[1] + m[3 * i + 2] * v[2];
}
inline void mat3t_vec(const double* m, const double* v, double* o) {
    for (int i = 0; i < 3; ++i) o[i] = m[0 + i] * v[0] + m[3 + i] * v[1] + m[6 + i] * v[2];
}

// sfm-lite/src/geom.rs:28-42  Cam::normalize
inline void cam_normalize(double f, double cx, double cy, double k, double u, double v, double* o) {
    double xn = (u - cx) / f;
    double yn = (v - cy) / f;
    for (int it = 0; it < 2; ++it) {
        double r2 = xn * xn + yn * yn;
        double d = 1.0 + k * r2;
        if (std::fabs(d) < 1e-12) break;
        xn = (u - cx) / (f * d);
        yn = (v - cy) / (f * d);
    }
    o[0] = xn;
    o[1] = yn;
}

// sfm-lite/src/geom.rs:64-75  Pose::project
inline bool pose_project(const rcmvs_view& v, const double* x, double* uv) {
    double xc[3];
    mat3_vec(v.R, x, xc);
    for (int i = 0; i < 3; ++i) xc[i] = xc[i] + v.t[i];
    double z = xc[2];
    if (z <= 1e-9) return false;
    double xn = xc[0] / z;
    double yn = xc[1] / z;
    double r2 = xn * xn + yn * yn;
    double d = 1.0 + v.k * r2;
    uv[0] = v.f * xn * d + v.cx;
    uv[1] = v.f * yn * d + v.cy;
    return true;
}

// ---------------------------------------------------------------- stereo
// mvs/src/stereo.rs:84-96  SourceCtx
struct SourceCtx {
    const uint64_t* census;
    int32_t w, h;
    float f, cx, cy, k;
    float rs[9];
    float ts[3];
};

// mvs/src/stereo.rs:103-111  RefWorkspace
struct RefWorkspace {
    int32_t w, h;
    const uint64_t* census;
    std::vector<float> rx, ry;
    std::vector<SourceCtx> sources;
    float zmin, zmax;
};

const float BITS = 48.0f;  // stereo.rs:40
const int32_t WIN = 2;     // stereo.rs:41

// mvs/src/stereo.rs:131-132 (rs64 = R_s R_r^T, ts64 = t_s - rs64 t_r)
void rel_pose(const rcmvs_view& r, const rcmvs_view& s, float* rs, float* ts) {
    double rs64[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            rs64[3 * i + j] = s.R[3 * i + 0] * r.R[3 * j + 0] + s.R[3 * i + 1] * r.R[3 * j + 1] +
                              s.R[3 * i + 2] * r.R[3 * j + 2];
    double rt[3];
    mat3_vec(rs64, r.t, rt);
    for (int i = 0; i < 9; ++i) rs[i] = (float)rs64[i];
    for (int i = 0; i < 3; ++i) ts[i] = (float)(s.t[i] - rt[i]);
}

// mvs/src/stereo.rs:114-151  RefWorkspace::new
void ws_init(RefWorkspace& ws, const rcmvs_view* views, const std::vector<const uint64_t*>& census,
             int ref_idx, const int32_t* srcs, int n_src, double zmin, double zmax) {
    const rcmvs_view& r = views[ref_idx];
    ws.w = r.w;
    ws.h = r.h;
    ws.census = census[ref_idx];
    size_t n = (size_t)r.w * r.h;
    ws.rx.assign(n, 0.f);
    ws.ry.assign(n, 0.f);
    for (int32_t y = 0; y < r.h; ++y)
        for (int32_t x = 0; x < r.w; ++x) {
            double c[2];
            cam_normalize(r.f, r.cx, r.cy, r.k, (double)x, (double)y, c);
            size_t i = (size_t)y * r.w + x;
            ws.rx[i] = (float)c[0];
            ws.ry[i] = (float)c[1];
        }
    ws.sources.clear();
    for (int s = 0; s < n_src; ++s) {
        const rcmvs_view& sv = views[srcs[s]];
        SourceCtx sc;
        sc.census = census[srcs[s]];
        sc.w = sv.w;
        sc.h = sv.h;
        sc.f = (float)sv.f;
        sc.cx = (float)sv.cx;
        sc.cy = (float)sv.cy;
        sc.k = (float)sv.k;
        rel_pose(r, sv, sc.rs, sc.ts);
        ws.sources.push_back(sc);
    }
    ws.zmin = (float)zmin;
    ws.zmax = (float)zmax;
}

struct Work {
    uint64_t evals = 0, rows = 0;
};

// mvs/src/stereo.rs:158-228  plane_cost.  hsum (nullable) adds the integer
// Hamming sum (48 per invalid term) — a diagnostic with no reference
// counterpart that does not change the float result.
float plane_cost(const RefWorkspace& ws, int32_t px, int32_t py, float nx, float ny, float nz, float d,
                 float hint, Work* wk, int32_t* hsum) {
    const int32_t w = ws.w, h = ws.h;
    const float nsrc = (float)ws.sources.size();
    const float span = (float)(WIN * 2 + 1);
    const float total = span * span * nsrc;
    float sum = 0.f;
    bool aborted = false;
    int32_t hs = 0;
    if (wk) wk->evals++;
    for (size_t si = 0; si < ws.sources.size() && !aborted; ++si) {
        const SourceCtx& s = ws.sources[si];
        const int32_t sw = s.w, sh = s.h;
        const float f = s.f, cx = s.cx, cy = s.cy, k = s.k;
        const float* rs = s.rs;
        const float* ts = s.ts;
        for (int32_t dy = -WIN; dy <= WIN; ++dy) {
            int32_t yy = py + dy;
            int32_t ycl = clampi(yy, 0, h - 1);
            for (int32_t dx = -WIN; dx <= WIN; ++dx) {
                int32_t xx = px + dx;
                int32_t xcl = clampi(xx, 0, w - 1);
                size_t j = (size_t)ycl * w + xcl;
                float xo = ws.rx[j];
                float yo = ws.ry[j];
                float denom = nx * xo + ny * yo + nz;
                if (denom < 0.05f) {
                    sum += 1.0f;
                    hs += 48;
                    continue;
                }
                float z = d / denom;
                float xr = z * xo;
                float yr = z * yo;
                float xs = rs[0] * xr + rs[1] * yr + rs[2] * z + ts[0];
                float ys = rs[3] * xr + rs[4] * yr + rs[5] * z + ts[1];
                float zs = rs[6] * xr + rs[7] * yr + rs[8] * z + ts[2];
                if (zs < 1e-3f) {
                    sum += 1.0f;
                    hs += 48;
                    continue;
                }
                float xn = xs / zs;
                float yn = ys / zs;
                float dist = 1.0f + k * (xn * xn + yn * yn);
                int32_t u = orc_f32_to_i32(f * xn * dist + cx);
                int32_t v = orc_f32_to_i32(f * yn * dist + cy);
                if (u < 0 || v < 0 || u >= sw || v >= sh) {
                    sum += 1.0f;
                    hs += 48;
                    continue;
                }
                uint64_t csrc = s.census[(size_t)v * sw + u];
                uint64_t cref = ws.census[j];
                int pc = __builtin_popcountll(cref ^ csrc);
                hs += pc;
                sum += (float)pc / BITS;
            }
            if (wk) wk->rows++;
            float rows_done = (float)(dy + WIN + 1);
            if (sum / (rows_done * span * (float)(si + 1)) > hint + 0.12f) {
                aborted = true;
                break;
            }
        }
    }
    if (hsum) *hsum = hs;
    if (aborted) return 1e9f;
    return sum / total;
}

// mvs/src/stereo.rs:24-31
struct Plane {
    float nx, ny, nz, z, cost;
};

std::vector<const uint64_t*> census_for(const rcmvs_view* views, int n_views,
                                        const std::vector<int>& needed,
                                        std::vector<std::vector<uint64_t>>& store) {
    store.assign(n_views, {});
    std::vector<const uint64_t*> ptrs(n_views, nullptr);
    for (int v : needed) {
        if (!ptrs[v]) {
            store[v].resize((size_t)views[v].w * views[v].h);
            orc_census_map(views[v].gray, views[v].w, views[v].h, store[v].data());
            ptrs[v] = store[v].data();
        }
    }
    return ptrs;
}

bool check_views(const rcmvs_view* views, int32_t n_views, int32_t ref_idx, const int32_t* srcs,
                 int32_t n_src) {
    if (!views || n_views <= 0 || ref_idx < 0 || ref_idx >= n_views || n_src < 0) return false;
    if (n_src > 0 && !srcs) return false;
    for (int i = 0; i < n_src; ++i)
        if (srcs[i] < 0 || srcs[i] >= n_views) return false;
    for (int i = 0; i < n_views; ++i)
        if (views[i].w <= 0 || views[i].h <= 0) return false;
    return true;
}

}  // namespace

extern "C" {

// mvs/src/lib.rs:119-142  census_map (grey as u8/255 in f32, lib.rs:196)
void orc_census_map(const uint8_t* gray, int32_t w, int32_t h, uint64_t* out) {
    std::vector<float> g((size_t)w * h);
    for (size_t i = 0; i < g.size(); ++i) g[i] = (float)gray[i] / 255.0f;
    for (int32_t y = 0; y < h; ++y)
        for (int32_t x = 0; x < w; ++x) {
            float c = g[(size_t)y * w + x];
            uint64_t bits = 0;
            for (int32_t dy = -3; dy <= 3; ++dy)
                for (int32_t dx = -3; dx <= 3; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    int32_t xx = clampi(x + dx, 0, w - 1);
                    int32_t yy = clampi(y + dy, 0, h - 1);
                    uint64_t bit = (uint64_t)((dy + 3) * 7 + (dx + 3));
                    if (g[(size_t)yy * w + xx] < c) bits |= 1ull << bit;
                }
            out[(size_t)y * w + x] = bits;
        }
}

// mvs/src/stereo.rs:47-57  pixel_rng
uint64_t orc_pixel_rng(int32_t x, int32_t y, uint64_t salt) {
    uint64_t s = ((uint64_t)(int64_t)x * 0x9E3779B97F4A7C15ull) ^
                 ((uint64_t)(int64_t)y * 0xC2B2AE3D27D4EB4Full) ^ (salt * 0x165667B19E3779F9ull);
    s ^= s >> 30;
    s *= 0xBF58476D1CE4E5B9ull;
    s ^= s >> 27;
    s *= 0x94D049BB133111EBull;
    return s ^ (s >> 31);
}

// mvs/src/stereo.rs:59-67  next_u64 (xorshift64)
uint64_t orc_next_u64(uint64_t* s) {
    uint64_t x = *s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *s = x;
    return x;
}

// mvs/src/stereo.rs:69-72
float orc_uniform(uint64_t* s) { return (float)(orc_next_u64(s) >> 40) / (float)(1ull << 24); }

// mvs/src/stereo.rs:74-78  (operands evaluate left to right)
float orc_gauss(uint64_t* s) {
    float a = orc_uniform(s);
    float b = orc_uniform(s);
    float c = orc_uniform(s);
    return a + b + c - 1.5f;
}

// Rust `f32 as i32`: truncate toward zero, saturate, NaN -> 0.
int32_t orc_f32_to_i32(float v) {
    if (std::isnan(v)) return 0;
    if (v >= 2147483648.0f) return INT32_MAX;
    if (v < -2147483648.0f) return INT32_MIN;
    return (int32_t)v;
}

void orc_cam_normalize(double f, double cx, double cy, double k, double u, double v, double* out2) {
    cam_normalize(f, cx, cy, k, u, v, out2);
}

void orc_rays(const rcmvs_view* v, float* rx, float* ry) {
    for (int32_t y = 0; y < v->h; ++y)
        for (int32_t x = 0; x < v->w; ++x) {
            double c[2];
            cam_normalize(v->f, v->cx, v->cy, v->k, (double)x, (double)y, c);
            rx[(size_t)y * v->w + x] = (float)c[0];
            ry[(size_t)y * v->w + x] = (float)c[1];
        }
}

void orc_rel_pose(const rcmvs_view* ref, const rcmvs_view* src, float* rs9, float* ts3) {
    rel_pose(*ref, *src, rs9, ts3);
}

int orc_plane_cost_field(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                         const int32_t* srcs, int32_t n_src, const float* planes,
                         const float* hints, float* cost_out, int32_t* hsum_out,
                         int32_t nthreads) {
    if (!check_views(views, n_views, ref_idx, srcs, n_src) || !planes || !hints || !cost_out)
        return RCMVS_E_ARG;
    std::vector<int> needed{ref_idx};
    for (int i = 0; i < n_src; ++i) needed.push_back(srcs[i]);
    std::vector<std::vector<uint64_t>> store;
    auto cen = census_for(views, n_views, needed, store);
    RefWorkspace ws;
    ws_init(ws, views, cen, ref_idx, srcs, n_src, 0.0, 0.0);
    const int32_t w = ws.w, h = ws.h;
    par_for(h, nthreads, [&](int64_t y, int) {
        for (int32_t x = 0; x < w; ++x) {
            size_t i = (size_t)y * w + x;
            int32_t hs = 0;
            cost_out[i] = plane_cost(ws, x, (int32_t)y, planes[4 * i], planes[4 * i + 1],
                                     planes[4 * i + 2], planes[4 * i + 3], hints[i], nullptr, &hs);
            if (hsum_out) hsum_out[i] = hs;
        }
    });
    return RCMVS_OK;
}

}  // extern "C"

namespace {

// Learned-proposal seeding of the init (no reference counterpart): the
// quarter-resolution predictions of the reference view (wq*hq cells of 16
// f32: t, normal xyz, confidence logit, ...) and the selection parameters.
struct Seed {
    const float* pred;
    float logit_thr;  // confident iff logit >= logit_thr
    int32_t n_local;
    float span;
    bool sweep_seeded;  // a seeded pixel also runs the sweep (RCMVS_FLAG_SEED_AND_SWEEP)
    uint64_t seeded = 0;
};

// Plane-sweep init of one pixel (stereo.rs:247-269).  `start` (nullable) is
// a plane already scored for the pixel: the sweep then begins with its cost
// as the best so far and keeps it unless a hypothesis is strictly cheaper.
Plane sweep_init(const RefWorkspace& ws, int32_t x, int32_t y, int32_t nh, float inv_min, float inv_max, Work* wk,
                 const Plane* start = nullptr) {
    float best_c = start ? start->cost : INFINITY;
    float best_d = 0.f;
    bool improved = false;
    for (int32_t hi = 0; hi < nh; ++hi) {
        float inv = inv_min + (inv_max - inv_min) * (float)hi / (float)(nh - 1);
        float d = 1.0f / inv;
        float c = plane_cost(ws, x, y, 0.0f, 0.0f, 1.0f, d, best_c + 0.02f, wk, nullptr);
        if (c < best_c) {
            best_c = c;
            best_d = d;
            improved = true;
        }
    }
    if (start && !improved) return *start;
    return Plane{0.0f, 0.0f, 1.0f, best_d, std::fmin(best_c, 1.0f)};
}

// Learned init of one pixel, as the library's init_learned_rows_kernel
// computes it: the pixel's quarter cell (min(x/4, wq-1), min(y/4, hq-1))
// proposes a plane when its logit >= logit_thr and its normal is not
// degenerate; the predicted inverse depth t (a fraction of [1/zmax, 1/zmin])
// is placed on the ray of the cell's anchor pixel (4qx+1, 4qy+1), so every
// pixel of the cell gets the same plane (n, d).  n_local planes spread over
// +-span/2 around t are scored with plane_cost and the sweep's hint rule;
// one that fails the stereo gates (n.ray >= 0.1 at the pixel and the anchor,
// positive inverse depth, depth in [zmin/2, 2 zmax]) is skipped.  A pixel
// without a usable proposal runs the plane sweep.  Returns whether the
// pixel was seeded.  With sweep_seeded a seeded pixel then runs the sweep
// from its proposal's cost (the GPU's phase 2 does the same).
bool learned_init(const RefWorkspace& ws, const Seed& sd, int32_t x, int32_t y, int32_t nh, float inv_min,
                  float inv_max, Work* wk, Plane* out) {
    const int32_t w = ws.w, h = ws.h;
    const int32_t wq = w >> 2, hq = h >> 2;
    const size_t i = (size_t)y * w + x;
    const float zlo = ws.zmin * 0.5f, zhi = ws.zmax * 2.0f;
    const float span_inv = inv_max - inv_min;
    if (wq > 0 && hq > 0) {
        const int32_t qx = std::min(x >> 2, wq - 1), qy = std::min(y >> 2, hq - 1);
        const float* o = sd.pred + ((size_t)qy * wq + qx) * 16;
        const float len = std::sqrt(o[1] * o[1] + o[2] * o[2] + o[3] * o[3]);
        if (o[4] >= sd.logit_thr && len > 1e-6f) {
            const float pnx = o[1] / len, pny = o[2] / len, pnz = o[3] / len;
            const float pa = pnx * ws.rx[i] + pny * ws.ry[i] + pnz;
            const size_t ia = (size_t)(4 * qy + 1) * w + (4 * qx + 1);
            const float pac = pnx * ws.rx[ia] + pny * ws.ry[ia] + pnz;
            if (pa >= 0.1f && pac >= 0.1f) {
                const float t0 = o[0];
                float best_c = INFINITY;
                Plane best{0.0f, 0.0f, 1.0f, 0.0f, 0.0f};
                bool any = false;
                for (int32_t k = 0; k < sd.n_local; ++k) {
                    const float tk = t0 + sd.span * ((float)k / (float)std::max(sd.n_local - 1, 1) - 0.5f);
                    const float inv = inv_min + tk * span_inv;
                    if (!(inv > 0.f)) continue;
                    const float z = 1.0f / inv;   // depth on the anchor ray
                    const float dcell = z * pac;  // the cell's plane offset
                    const float zi = dcell / pa;  // depth on this pixel's ray
                    if (!(zi >= zlo && zi <= zhi)) continue;
                    any = true;
                    const float c = plane_cost(ws, x, y, pnx, pny, pnz, dcell, best_c + 0.02f, wk, nullptr);
                    if (c < best_c) {
                        best_c = c;
                        best = Plane{pnx, pny, pnz, zi, 0.0f};
                    }
                }
                if (any) {
                    best.cost = std::fmin(best_c, 1.0f);
                    *out = sd.sweep_seeded ? sweep_init(ws, x, y, nh, inv_min, inv_max, wk, &best) : best;
                    return true;
                }
            }
        }
    }
    *out = sweep_init(ws, x, y, nh, inv_min, inv_max, wk);
    return false;
}

// stereo::estimate_depth, with the init optionally seeded (sd != nullptr)
// and the passes optionally left out (RCMVS_FLAG_INIT_ONLY).
int estimate_impl(const rcmvs_view* views, int32_t n_views, int32_t ref_idx, const int32_t* srcs, int32_t n_src,
                  double zmin, double zmax, const rcmvs_options* opts, float* depth_out, float* cost_out,
                  float* normal_out, int32_t nthreads, uint64_t* work_out, Seed* sd) {
    if (!check_views(views, n_views, ref_idx, srcs, n_src) || !opts || !depth_out || !cost_out ||
        opts->passes > RCMVS_MAX_PASSES)
        return RCMVS_E_ARG;
    std::vector<int> needed{ref_idx};
    for (int i = 0; i < n_src; ++i) needed.push_back(srcs[i]);
    std::vector<std::vector<uint64_t>> store;
    auto cen = census_for(views, n_views, needed, store);
    RefWorkspace ws;
    ws_init(ws, views, cen, ref_idx, srcs, n_src, zmin, zmax);
    const int32_t w = ws.w, h = ws.h;
    const size_t npx = (size_t)w * h;
    int nt = nthreads <= 0 ? (int)std::thread::hardware_concurrency() : nthreads;
    if (nt < 1) nt = 1;
    std::vector<Work> work(nt);

    // ---- plane-sweep init (stereo.rs:247-269)
    const float inv_min = 1.0f / ws.zmax;
    const float inv_max = 1.0f / ws.zmin;
    const int32_t nh = (int32_t)std::max<uint32_t>(opts->num_hyp, 2u);
    std::vector<Plane> prev(npx);
    std::vector<uint64_t> seeded(nt, 0);
    par_for(h, nt, [&](int64_t y, int t) {
        for (int32_t x = 0; x < w; ++x) {
            Plane& p = prev[(size_t)y * w + x];
            if (sd)
                seeded[t] += learned_init(ws, *sd, x, (int32_t)y, nh, inv_min, inv_max, &work[t], &p);
            else
                p = sweep_init(ws, x, (int32_t)y, nh, inv_min, inv_max, &work[t]);
        }
    });
    if (sd)
        for (uint64_t c : seeded) sd->seeded += c;

    // ---- double-buffered passes (stereo.rs:271-371); none with RCMVS_FLAG_INIT_ONLY
    // the passes option (an extension; 0 = the reference's 2 * max(sweeps, 1))
    const uint64_t n_passes = (opts->flags & RCMVS_FLAG_INIT_ONLY) ? 0
                              : opts->passes                     ? (uint64_t)opts->passes
                                                                 : (uint64_t)std::max<uint32_t>(opts->sweeps, 1u) * 2;
    std::vector<Plane> next = prev;
    const float zlo = ws.zmin * 0.5f, zhi = ws.zmax * 2.0f;
    for (uint64_t pass = 0; pass < n_passes; ++pass) {
        const float t = (float)pass / (float)n_passes;
        const float sig_inv = 0.02f * powf(0.28f, t * 4.0f);
        const float sig_n = 0.30f * powf(0.42f, t * 4.0f);
        next = prev;
        par_for(h, nt, [&](int64_t yy64, int tid) {
            const int32_t y = (int32_t)yy64;
            for (int32_t x = 0; x < w; ++x) {
                const size_t i = (size_t)y * w + x;
                uint64_t seed = orc_pixel_rng(x, y, pass + 7);
                const Plane cur = prev[i];
                float best_c = cur.cost;
                float bn[3] = {cur.nx, cur.ny, cur.nz};
                float bd = cur.z * (bn[0] * ws.rx[i] + bn[1] * ws.ry[i] + bn[2]);
                static const int32_t NB[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
                for (int q = 0; q < 4; ++q) {
                    int32_t xx = x + NB[q][0], yy = y + NB[q][1];
                    if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                    size_t j = (size_t)yy * w + xx;
                    const Plane nb = prev[j];
                    float a_nb = nb.nx * ws.rx[j] + nb.ny * ws.ry[j] + nb.nz;
                    if (a_nb < 0.1f) continue;
                    float d_plane = nb.z * a_nb;
                    float a_here = nb.nx * ws.rx[i] + nb.ny * ws.ry[i] + nb.nz;
                    if (a_here < 0.1f) continue;
                    float zcand = d_plane / a_here;
                    if (!(zlo <= zcand && zcand <= zhi)) continue;
                    float c = plane_cost(ws, x, y, nb.nx, nb.ny, nb.nz, d_plane, best_c + 0.02f,
                                         &work[tid], nullptr);
                    if (c < best_c) {
                        best_c = c;
                        bn[0] = nb.nx;
                        bn[1] = nb.ny;
                        bn[2] = nb.nz;
                        bd = d_plane;
                    }
                }
                for (int r = 0; r < 3; ++r) {
                    float inv = 1.0f / std::fmax(cur.z, 1e-6f);
                    float inv_new = inv + sig_inv * (inv_max - inv_min) * orc_gauss(&seed);
                    if (inv_new <= 0.0f) continue;
                    float zcand = 1.0f / inv_new;
                    if (!(zlo <= zcand && zcand <= zhi)) continue;
                    float nnx = cur.nx + sig_n * orc_gauss(&seed);
                    float nny = cur.ny + sig_n * orc_gauss(&seed);
                    float nnz = cur.nz + sig_n * orc_gauss(&seed);
                    float len = std::sqrt(nnx * nnx + nny * nny + nnz * nnz);
                    if (len < 1e-6f) continue;
                    nnx = nnx / len;
                    nny = nny / len;
                    nnz = nnz / len;
                    float a_here = nnx * ws.rx[i] + nny * ws.ry[i] + nnz;
                    if (a_here < 0.1f) continue;
                    float d_plane = zcand * a_here;
                    float c = plane_cost(ws, x, y, nnx, nny, nnz, d_plane, best_c + 0.02f, &work[tid],
                                         nullptr);
                    if (c < best_c) {
                        best_c = c;
                        bn[0] = nnx;
                        bn[1] = nny;
                        bn[2] = nnz;
                        bd = d_plane;
                    }
                }
                if (best_c < cur.cost) {
                    float a_here = bn[0] * ws.rx[i] + bn[1] * ws.ry[i] + bn[2];
                    if (a_here > 0.05f) {
                        float z_new = bd / a_here;
                        next[i] = Plane{bn[0], bn[1], bn[2], z_new, std::fmin(best_c, 1.0f)};
                    }
                }
            }
        });
        std::swap(prev, next);
    }

    // ---- gate (stereo.rs:373-393)
    for (size_t i = 0; i < npx; ++i) {
        Plane& p = prev[i];
        int tex = __builtin_popcountll(ws.census[i]);
        bool textured = tex >= 4 && tex <= 44;
        bool ok = textured && p.cost < opts->cost_thr && p.z > ws.zmin * 0.5f && p.z < ws.zmax * 2.0f;
        if (!ok) p.z = 0.0f;
        depth_out[i] = p.z;
        cost_out[i] = p.cost;
        if (normal_out) {
            normal_out[3 * i] = p.nx;
            normal_out[3 * i + 1] = p.ny;
            normal_out[3 * i + 2] = p.nz;
        }
    }
    if (work_out) {
        work_out[0] = work_out[1] = 0;
        for (auto& wk : work) {
            work_out[0] += wk.evals;
            work_out[1] += wk.rows;
        }
    }
    return RCMVS_OK;
}

}  // namespace

extern "C" {

// mvs/src/stereo.rs:234-394  estimate_depth
int orc_estimate_depth(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                       const int32_t* srcs, int32_t n_src, double zmin, double zmax,
                       const rcmvs_options* opts, float* depth_out, float* cost_out,
                       float* normal_out, int32_t nthreads, uint64_t* work_out) {
    return estimate_impl(views, n_views, ref_idx, srcs, n_src, zmin, zmax, opts, depth_out, cost_out, normal_out,
                         nthreads, work_out, nullptr);
}

int orc_estimate_depth_seeded(const rcmvs_view* views, int32_t n_views, int32_t ref_idx,
                              const int32_t* srcs, int32_t n_src, double zmin, double zmax,
                              const rcmvs_options* opts, const float* pred, float conf_thr,
                              int32_t n_local, float span, float* depth_out, float* cost_out,
                              float* normal_out, int32_t nthreads, uint64_t* seeded_out) {
    if (!pred || n_local < 1 || n_local > 256 || !(span >= 0.f && span <= 1.f) || std::isnan(conf_thr))
        return RCMVS_E_ARG;
    Seed sd{pred, orc_logit_threshold(conf_thr), n_local, span, (opts->flags & RCMVS_FLAG_SEED_AND_SWEEP) != 0};
    const int rc = estimate_impl(views, n_views, ref_idx, srcs, n_src, zmin, zmax, opts, depth_out, cost_out,
                                 normal_out, nthreads, nullptr, &sd);
    if (seeded_out) *seeded_out = sd.seeded;
    return rc;
}

// The confidence test sigmoid(logit) >= conf_thr as a logit threshold,
// ln(c / (1 - c)) in f64 rounded to f32 (-inf for c <= 0, +inf for c >= 1).
float orc_logit_threshold(float conf_thr) {
    if (!(conf_thr > 0.0f)) return -INFINITY;
    if (!(conf_thr < 1.0f)) return INFINITY;
    const double c = (double)conf_thr;
    return (float)std::log(c / (1.0 - c));
}

// mvs/src/fuse.rs:32-62  sample_depth
static double sample_depth(const float* depth, int32_t w, int32_t h, double u, double v) {
    int32_t u0 = f64_to_i32(std::floor(u));
    int32_t v0 = f64_to_i32(std::floor(v));
    // fuse.rs:37 tests `u0 + 1 >= w`; written without the i32 overflow at
    // u0 = INT_MAX (a saturated projection), where the reference would wrap
    // and then panic on the slice index.  Such points count as off-image.
    if (u0 < 0 || v0 < 0 || u0 >= w - 1 || v0 >= h - 1) return 0.0;
    float fx = (float)(u - (double)u0);
    float fy = (float)(v - (double)v0);
    auto idx = [&](int32_t x, int32_t y) { return depth[(size_t)y * w + x]; };
    float ds[4] = {idx(u0, v0), idx(u0 + 1, v0), idx(u0, v0 + 1), idx(u0 + 1, v0 + 1)};
    float wt[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
    float acc = 0.f, wsum = 0.f;
    for (int q = 0; q < 4; ++q)
        if (ds[q] > 0.0f) {
            acc += ds[q] * wt[q];
            wsum += wt[q];
        }
    if (wsum > 1e-6f) return (double)(acc / wsum);
    return 0.0;
}

// mvs/src/fuse.rs:72-92: robust sparse bounding-box diagonal -> voxel cell
static double voxel_cell(const double* sparse_xyz, uint64_t n_sparse, double voxel_rel) {
    double ext[3];
    for (int a = 0; a < 3; ++a) {
        std::vector<double> ax(n_sparse);
        for (uint64_t p = 0; p < n_sparse; ++p) ax[p] = sparse_xyz[3 * p + a];
        std::sort(ax.begin(), ax.end());
        size_t len = ax.size();
        size_t ilo = std::min((size_t)((double)len * 0.02), len - 1);
        size_t ihi = std::min((size_t)((double)len * 0.98), len - 1);
        ext[a] = ax[ihi] - ax[ilo];
    }
    double diag = std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]);
    return std::fmax(diag * voxel_rel, 1e-9);
}

using Cand = std::array<double, 6>;  // averaged point, reference colour

// mvs/src/fuse.rs:96-167 for the views v with a depth map and ref_mask[v]
// (every such view when ref_mask is NULL): per view, its candidates in
// pixel order.
static void fuse_candidates(const rcmvs_view* views, int32_t n_views, const float* const* depth_maps,
                            const int32_t* order_offsets, const int32_t* order, const uint8_t* ref_mask,
                            const rcmvs_options* opts, std::vector<std::vector<Cand>>& per_view, int32_t nthreads) {
    per_view.assign(n_views, {});
    par_for(n_views, nthreads, [&](int64_t ri, int) {
        const float* dm = depth_maps[ri];
        if (!dm || (ref_mask && !ref_mask[ri])) return;
        const rcmvs_view& v = views[ri];
        auto& out = per_view[ri];
        for (int32_t py = 0; py < v.h; ++py)
            for (int32_t px = 0; px < v.w; ++px) {
                size_t i = (size_t)py * v.w + px;
                double zr = (double)dm[i];
                if (zr <= 0.0) continue;
                double nrm[2];
                cam_normalize(v.f, v.cx, v.cy, v.k, (double)px, (double)py, nrm);
                double xr[3] = {nrm[0] * zr, nrm[1] * zr, 1.0 * zr};
                double d[3] = {xr[0] - v.t[0], xr[1] - v.t[1], xr[2] - v.t[2]};
                double xw[3];
                mat3t_vec(v.R, d, xw);
                double acc[3] = {xw[0], xw[1], xw[2]};
                size_t n_cons = 0;
                for (int32_t q = order_offsets[ri]; q < order_offsets[ri + 1]; ++q) {
                    const rcmvs_view& sv = views[order[q]];
                    double xs[3];
                    mat3_vec(sv.R, xw, xs);
                    for (int a = 0; a < 3; ++a) xs[a] = xs[a] + sv.t[a];
                    if (xs[2] <= 1e-6) continue;
                    double uv[2];
                    if (!pose_project(sv, xw, uv)) continue;
                    double zs = sample_depth(depth_maps[order[q]], sv.w, sv.h, uv[0], uv[1]);
                    if (zs <= 0.0) continue;
                    double rel = std::fabs((xs[2] - zs) / xs[2]);
                    if (rel < opts->depth_diff) {
                        double ns[2];
                        cam_normalize(sv.f, sv.cx, sv.cy, sv.k, uv[0], uv[1], ns);
                        double xs2[3] = {ns[0] * zs, ns[1] * zs, 1.0 * zs};
                        double d2[3] = {xs2[0] - sv.t[0], xs2[1] - sv.t[1], xs2[2] - sv.t[2]};
                        double xw2[3];
                        mat3t_vec(sv.R, d2, xw2);
                        if (opts->reproj_px > 0.0) {
                            double ruv[2];
                            if (!pose_project(v, xw2, ruv)) continue;
                            double ex = ruv[0] - (double)px, ey = ruv[1] - (double)py;
                            if (!(std::sqrt(ex * ex + ey * ey) <= opts->reproj_px)) continue;
                        }
                        for (int a = 0; a < 3; ++a) acc[a] += xw2[a];
                        ++n_cons;
                    }
                }
                if (n_cons < opts->min_consistent) continue;
                double m = (double)(n_cons + 1);
                out.push_back(Cand{acc[0] / m, acc[1] / m, acc[2] / m, (double)v.rgb[3 * i],
                                   (double)v.rgb[3 * i + 1], (double)v.rgb[3 * i + 2]});
            }
    });
}

// mvs/src/fuse.rs:176-214: voxel dedup, members accumulated in the order
// given (the reference's view-then-pixel order); output in key order.
static int fuse_reduce(const std::vector<const Cand*>& cands, double cell, double** xyz_out, uint8_t** rgb_out,
                       uint64_t* n_out) {
    struct Fused {
        double x = 0, y = 0, z = 0;
        uint16_t r = 0, g = 0, b = 0;
        uint32_t n = 0;
    };
    std::map<std::tuple<int64_t, int64_t, int64_t>, Fused> vox;
    for (const Cand* pp : cands) {
        const Cand& p = *pp;
        auto key = std::make_tuple(f64_to_i64(std::floor(p[0] / cell)), f64_to_i64(std::floor(p[1] / cell)),
                                   f64_to_i64(std::floor(p[2] / cell)));
        Fused& e = vox[key];
        e.x += p[0];
        e.y += p[1];
        e.z += p[2];
        e.r = (uint16_t)(e.r + (uint16_t)p[3]);
        e.g = (uint16_t)(e.g + (uint16_t)p[4]);
        e.b = (uint16_t)(e.b + (uint16_t)p[5]);
        e.n += 1;
    }
    uint64_t n = vox.size();
    double* xyz = (double*)std::malloc(sizeof(double) * 3 * (n ? n : 1));
    uint8_t* rgb = (uint8_t*)std::malloc(3 * (n ? n : 1));
    if (!xyz || !rgb) {
        std::free(xyz);
        std::free(rgb);
        return RCMVS_E_NOMEM;
    }
    uint64_t o = 0;
    for (auto& kv : vox) {
        const Fused& e = kv.second;
        double nn = (double)e.n;
        xyz[3 * o] = e.x / nn;
        xyz[3 * o + 1] = e.y / nn;
        xyz[3 * o + 2] = e.z / nn;
        rgb[3 * o] = f64_to_u8(std::round((double)e.r / nn));
        rgb[3 * o + 1] = f64_to_u8(std::round((double)e.g / nn));
        rgb[3 * o + 2] = f64_to_u8(std::round((double)e.b / nn));
        ++o;
    }
    *xyz_out = xyz;
    *rgb_out = rgb;
    *n_out = n;
    return RCMVS_OK;
}

static int check_fuse_args(const rcmvs_view* views, int32_t n_views, const float* const* depth_maps,
                           const int32_t* order_offsets, const int32_t* order) {
    for (int v = 0; v < n_views; ++v) {
        for (int32_t q = order_offsets[v]; q < order_offsets[v + 1]; ++q)
            if (order[q] < 0 || order[q] >= n_views || !depth_maps[order[q]]) return RCMVS_E_ARG;
        if (depth_maps[v] && !views[v].rgb) return RCMVS_E_ARG;
    }
    return RCMVS_OK;
}

// mvs/src/fuse.rs:64-215  fuse_depth_maps (+ the reprojection extension,
// off unless opts->reproj_px > 0)
int orc_fuse_depth_maps(const rcmvs_view* views, int32_t n_views, const float* const* depth_maps,
                        const int32_t* order_offsets, const int32_t* order,
                        const double* sparse_xyz, uint64_t n_sparse, const rcmvs_options* opts,
                        double** xyz_out, uint8_t** rgb_out, uint64_t* n_out,
                        uint64_t* n_candidates_out, int32_t nthreads) {
    if (!views || n_views <= 0 || !depth_maps || !order_offsets || !opts || !xyz_out || !rgb_out ||
        !n_out || n_sparse == 0 || !sparse_xyz)
        return RCMVS_E_ARG;
    if (check_fuse_args(views, n_views, depth_maps, order_offsets, order)) return RCMVS_E_ARG;
    const double cell = voxel_cell(sparse_xyz, n_sparse, opts->voxel_rel);
    std::vector<std::vector<Cand>> per_view;
    fuse_candidates(views, n_views, depth_maps, order_offsets, order, nullptr, opts, per_view, nthreads);
    std::vector<const Cand*> all;
    for (auto& vp : per_view)
        for (auto& p : vp) all.push_back(&p);
    if (n_candidates_out) *n_candidates_out = all.size();
    return fuse_reduce(all, cell, xyz_out, rgb_out, n_out);
}

int orc_fuse_candidates(const rcmvs_view* views, int32_t n_views, const float* const* depth_maps,
                        const int32_t* order_offsets, const int32_t* order, const uint8_t* ref_mask,
                        const rcmvs_options* opts, double** xyz_out, uint8_t** rgb_out, uint64_t* n_out,
                        uint64_t* per_view_out, int32_t nthreads) {
    if (!views || n_views <= 0 || !depth_maps || !order_offsets || !opts || !xyz_out || !rgb_out || !n_out)
        return RCMVS_E_ARG;
    if (check_fuse_args(views, n_views, depth_maps, order_offsets, order)) return RCMVS_E_ARG;
    std::vector<std::vector<Cand>> per_view;
    fuse_candidates(views, n_views, depth_maps, order_offsets, order, ref_mask, opts, per_view, nthreads);
    uint64_t n = 0;
    for (auto& vp : per_view) n += vp.size();
    double* xyz = (double*)std::malloc(sizeof(double) * 3 * (n ? n : 1));
    uint8_t* rgb = (uint8_t*)std::malloc(3 * (n ? n : 1));
    if (!xyz || !rgb) {
        std::free(xyz);
        std::free(rgb);
        return RCMVS_E_NOMEM;
    }
    uint64_t o = 0;
    for (int v = 0; v < n_views; ++v) {
        if (per_view_out) per_view_out[v] = per_view[v].size();
        for (const Cand& p : per_view[v]) {
            for (int a = 0; a < 3; ++a) {
                xyz[3 * o + a] = p[a];
                rgb[3 * o + a] = (uint8_t)p[3 + a];
            }
            ++o;
        }
    }
    *xyz_out = xyz;
    *rgb_out = rgb;
    *n_out = n;
    return RCMVS_OK;
}

int orc_fuse_reduce(const double* xyz, const uint8_t* rgb, uint64_t n, const double* sparse_xyz, uint64_t n_sparse,
                    const rcmvs_options* opts, double** xyz_out, uint8_t** rgb_out, uint64_t* n_out) {
    if ((n > 0 && (!xyz || !rgb)) || !sparse_xyz || n_sparse == 0 || !opts || !xyz_out || !rgb_out || !n_out)
        return RCMVS_E_ARG;
    std::vector<Cand> c(n);
    std::vector<const Cand*> all(n);
    for (uint64_t i = 0; i < n; ++i) {
        c[i] = Cand{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], (double)rgb[3 * i], (double)rgb[3 * i + 1],
                    (double)rgb[3 * i + 2]};
        all[i] = &c[i];
    }
    return fuse_reduce(all, voxel_cell(sparse_xyz, n_sparse, opts->voxel_rel), xyz_out, rgb_out, n_out);
}

void orc_free(void* p) { std::free(p); }

// mvs/src/fuse.rs:222-239  write_ply_binary
int orc_write_ply_binary(const char* path, const double* xyz, const uint8_t* rgb, uint64_t n) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return RCMVS_E_IO;
    std::fprintf(f,
                 "ply\nformat binary_little_endian 1.0\ncomment rustcolmap dense MVS fusion\n"
                 "element vertex %llu\nproperty float x\nproperty float y\nproperty float z\n"
                 "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n",
                 (unsigned long long)n);
    for (uint64_t i = 0; i < n; ++i) {
        float p[3] = {(float)xyz[3 * i], (float)xyz[3 * i + 1], (float)xyz[3 * i + 2]};
        std::fwrite(p, 4, 3, f);  // x86-64 is little-endian
        std::fwrite(rgb + 3 * i, 1, 3, f);
    }
    return std::fclose(f) == 0 ? RCMVS_OK : RCMVS_E_IO;
}

// mvs/src/fuse.rs:241-268  save_depth_vis (the image; the PNG encoding is
// the caller's).  lo_hi (nullable) receives the two percentiles.
void orc_depth_vis(const float* depth, int32_t w, int32_t h, uint8_t* out, float* lo_hi) {
    const size_t n = (size_t)w * h;
    std::vector<float> ds;
    for (size_t i = 0; i < n; ++i)
        if (depth[i] > 0.0f) ds.push_back(depth[i]);
    std::sort(ds.begin(), ds.end());  // partial_cmp order; no NaN passes z > 0
    float lo = 0.0f, hi = 1.0f;
    if (ds.size() >= 32) {
        lo = ds[(size_t)((double)ds.size() * 0.02)];
        hi = ds[(size_t)((double)ds.size() * 0.98) - 1];
    }
    const float range = std::max(hi - lo, 1e-9f);
    for (size_t i = 0; i < n; ++i) {
        const float z = depth[i];
        uint8_t val = 0;
        if (!(z <= 0.0f)) {
            float t = (z - lo) / range;
            if (t < 0.0f) t = 0.0f;          // f32::clamp(0.0, 1.0)
            else if (t > 1.0f) t = 1.0f;
            const float v = 255.0f * (1.0f - t);
            // `as u8`: truncation, saturating, NaN -> 0
            val = !(v > 0.0f) ? 0 : (v >= 255.0f ? 255 : (uint8_t)(int)v);
        }
        out[i] = val;
    }
    if (lo_hi) {
        lo_hi[0] = lo;
        lo_hi[1] = hi;
    }
}

// image 0.24 imageops::sample (the crate the reference resizes with at
// mvs/src/lib.rs:188-190; not in the reference tree): the taps of output
// sample o along an axis of n inputs resampled to m, Triangle filter
// (support 1, kernel |x| < 1 ? 1 - |x| : 0), weights normalised by their
// f32 sum.  Returns the first tap; ws gets the weights.
static uint32_t triangle_taps(uint32_t n, uint32_t m, uint32_t o, std::vector<float>& ws) {
    const float ratio = (float)n / (float)m;
    const float sratio = ratio < 1.0f ? 1.0f : ratio;
    const float src_support = 1.0f * sratio;
    float input = ((float)o + 0.5f) * ratio;
    int64_t left = (int64_t)std::floor(input - src_support);
    left = std::min(std::max(left, (int64_t)0), (int64_t)n - 1);
    int64_t right = (int64_t)std::ceil(input + src_support);
    right = std::min(std::max(right, left + 1), (int64_t)n);
    input = input - 0.5f;
    ws.clear();
    float sum = 0.0f;
    for (int64_t i = left; i < right; ++i) {
        const float x = ((float)i - input) / sratio;
        const float w = std::fabs(x) < 1.0f ? 1.0f - std::fabs(x) : 0.0f;
        ws.push_back(w);
        sum += w;
    }
    for (float& w : ws) w /= sum;
    return (uint32_t)left;
}

static uint8_t luma709(uint32_t r, uint32_t g, uint32_t b) {
    return (uint8_t)((2126u * r + 7152u * g + 722u * b) / 10000u);
}

void orc_resize_view(const uint8_t* img, int32_t w, int32_t h, int32_t channels, int32_t mw, int32_t mh,
                     uint8_t* gray, uint8_t* rgb) {
    const int nc = channels < 3 ? 1 : 3;  // colour channels; alpha is dropped
    const size_t n_out = (size_t)mw * mh;
    std::vector<uint8_t> px(n_out * nc);
    if (mw == w && mh == h) {  // lib.rs:188-192: the image as decoded
        for (size_t i = 0; i < n_out; ++i)
            for (int c = 0; c < nc; ++c) px[i * nc + c] = img[i * channels + c];
    } else {
        // vertical_sample: w columns x mh rows of f32
        std::vector<float> tmp((size_t)w * mh * nc), ws;
        for (int32_t oy = 0; oy < mh; ++oy) {
            const uint32_t top = triangle_taps((uint32_t)h, (uint32_t)mh, (uint32_t)oy, ws);
            for (int32_t x = 0; x < w; ++x)
                for (int c = 0; c < nc; ++c) {
                    float t = 0.0f;
                    for (size_t i = 0; i < ws.size(); ++i)
                        t += (float)img[(((size_t)top + i) * w + x) * channels + c] * ws[i];
                    tmp[((size_t)oy * w + x) * nc + c] = t;
                }
        }
        // horizontal_sample: clamp to [0, 255], round half away from zero
        for (int32_t ox = 0; ox < mw; ++ox) {
            const uint32_t first = triangle_taps((uint32_t)w, (uint32_t)mw, (uint32_t)ox, ws);
            for (int32_t y = 0; y < mh; ++y)
                for (int c = 0; c < nc; ++c) {
                    float t = 0.0f;
                    for (size_t i = 0; i < ws.size(); ++i) t += tmp[((size_t)y * w + first + i) * nc + c] * ws[i];
                    t = t < 0.0f ? 0.0f : (t > 255.0f ? 255.0f : t);
                    px[((size_t)y * mw + ox) * nc + c] = (uint8_t)std::round(t);
                }
        }
    }
    // to_luma8 / to_rgb8
    for (size_t i = 0; i < n_out; ++i) {
        const uint8_t* p = &px[i * nc];
        const uint8_t g = nc == 1 ? p[0] : luma709(p[0], p[1], p[2]);
        if (gray) gray[i] = g;
        if (rgb)
            for (int c = 0; c < 3; ++c) rgb[3 * i + c] = nc == 1 ? p[0] : p[c];
    }
}

// mvs/src/lib.rs:245-251  percentile
static double percentile(const std::vector<double>& s, double q) {
    if (s.empty()) return 0.0;
    double idx = std::round(((double)s.size() - 1.0) * q);
    idx = std::min(std::max(idx, 0.0), (double)s.size() - 1.0);
    return s[(size_t)idx];
}

// Host glue of run_mvs: lib.rs:224-243 covisibility, :253-282
// depth_range_for, :303-315 global depths, :326-342 sources, :398-418
// fusion order.  Ties in the count sort keep ascending view index (the
// reference's unstable sort is an insertion sort, hence stable, for <= 20
// candidates; beyond that its tie order is implementation-defined).
int orc_plan(const rcmvs_sparse* sp, const rcmvs_view* views, int32_t n_views,
             const rcmvs_options* opts, int32_t* src_offsets, int32_t* srcs, double* zrange,
             int32_t* fuse_offsets, int32_t* fuse_order) {
    if (!sp || !views || n_views <= 0 || !opts || !src_offsets || !srcs || !zrange ||
        !fuse_offsets || !fuse_order)
        return RCMVS_E_ARG;
    if (sp->n_points < 8) return RCMVS_E_ARG;  // lib.rs:310-315
    const int n = n_views;
    std::vector<double> global;
    for (uint64_t p = 0; p < sp->n_points; ++p) {
        const double* x = sp->xyz + 3 * p;
        global.push_back(std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]));
    }
    std::sort(global.begin(), global.end());
    std::vector<uint32_t> cov((size_t)n * n, 0);
    std::vector<std::vector<uint64_t>> pts_of_view(n);
    for (uint64_t p = 0; p < sp->n_points; ++p) {
        std::vector<int> ids;
        for (uint64_t q = sp->track_offsets[p]; q < sp->track_offsets[p + 1]; ++q) {
            int v = sp->track_views[q];
            if (v >= 0 && v < n) ids.push_back(v);
        }
        std::sort(ids.begin(), ids.end());
        ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
        for (int a : ids) {
            pts_of_view[a].push_back(p);
            for (int b : ids)
                if (a != b) cov[(size_t)a * n + b] += 1;
        }
    }
    auto ranked = [&](int i, bool need_depth, const std::vector<char>& has) {
        std::vector<std::pair<uint32_t, int>> o;
        for (int j = 0; j < n; ++j) {
            uint32_t c = cov[(size_t)i * n + j];
            if (c >= 10 && (!need_depth || has[j])) o.push_back({c, j});
        }
        std::stable_sort(o.begin(), o.end(), [](auto& a, auto& b) { return a.first > b.first; });
        return o;
    };
    std::vector<std::vector<int>> sources(n);
    std::vector<char> has(n, 0);
    int off = 0;
    for (int i = 0; i < n; ++i) {
        auto o = ranked(i, false, has);
        src_offsets[i] = off;
        for (size_t q = 0; q < o.size() && q < opts->num_sources; ++q) {
            sources[i].push_back(o[q].second);
            srcs[off++] = o[q].second;
        }
        has[i] = !sources[i].empty();
    }
    src_offsets[n] = off;
    for (int i = 0; i < n; ++i) {
        const rcmvs_view& v = views[i];
        std::vector<double> ds;
        for (uint64_t p : pts_of_view[i]) {
            double xc[3];
            mat3_vec(v.R, sp->xyz + 3 * p, xc);
            double z = xc[2] + v.t[2];
            if (z > 1e-6) ds.push_back(z);
        }
        const std::vector<double>* src = &global;
        if (ds.size() >= 8) {
            std::sort(ds.begin(), ds.end());
            src = &ds;
        }
        double lo = 0.0, hi = 0.0;
        if (src->size() >= 8) {
            lo = percentile(*src, 0.02);
            hi = percentile(*src, 0.98);
        }
        if (hi <= lo * 1.05 || lo <= 0.0) {
            double glo = percentile(global, 0.01), ghi = percentile(global, 0.99);
            zrange[2 * i] = std::fmax(glo * 0.7, 1e-3);
            zrange[2 * i + 1] = ghi * 1.4;
        } else {
            zrange[2 * i] = lo * 0.8;
            zrange[2 * i + 1] = hi * 1.25;
        }
    }
    off = 0;
    for (int i = 0; i < n; ++i) {
        auto o = ranked(i, true, has);
        std::vector<int> ord;
        for (auto& c : o) ord.push_back(c.second);
        const auto& s = sources[i];
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
            size_t pa = std::find(s.begin(), s.end(), a) - s.begin();
            size_t pb = std::find(s.begin(), s.end(), b) - s.begin();
            if (pa == s.size()) pa = SIZE_MAX;
            if (pb == s.size()) pb = SIZE_MAX;
            return pa < pb;
        });
        fuse_offsets[i] = off;
        for (int j : ord) fuse_order[off++] = j;
    }
    fuse_offsets[n] = off;
    return RCMVS_OK;
}

}  // extern "C"
