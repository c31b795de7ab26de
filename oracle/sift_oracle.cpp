// sift_oracle.cpp — CPU oracle for SIFT extraction (TEST INFRASTRUCTURE).
//
// Restates sfm-lite/src/sift.rs (extract_sift and its helpers) step by step:
// the Gaussian pyramid, DoG, 26-neighbour extrema with the quadratic fit,
// contrast and curvature rejection, 36-bin orientations and the 4x4x8
// descriptor, the response sort and the feature cap.  Used only by tests and
// the CPU leg of the benchmark as the checker; never linked into the product
// library.  The input is the image at working resolution (the resize is
// load-time work shared with the dense path).
//
// f32 and f64 arithmetic follows the reference's expression order (built with
// -ffp-contract=off); exp, atan2, cos and sin come from the host libm, as
// Rust's f64 methods do on Linux.  3x3 inverse: the cofactor form of
// nalgebra 0.32 (Cargo.lock) `try_inverse`.  PARITY UNPINNED: the Rust
// reference cannot be built here.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mvs_oracle.h"

namespace {

constexpr int NSPO = 3;           // sift.rs:14
constexpr double SIGMA0 = 1.6;    // sift.rs:15
constexpr double ASSUMED_BLUR = 0.5;
constexpr double EDGE_THR = 10.0;
constexpr int DESC_LEN = 128;
constexpr double PI = 3.14159265358979323846;

using Img = std::vector<float>;

// sift.rs:51-93
Img gauss_blur(const Img& src, size_t w, size_t h, double sigma) {
    if (sigma < 1e-4) return src;
    const size_t radius = (size_t)std::max(std::ceil(sigma * 3.0), 1.0);
    std::vector<double> kernel(2 * radius + 1);
    const double s2 = 2.0 * sigma * sigma;
    double sum = 0.0;
    for (size_t i = 0; i < kernel.size(); ++i) {
        const double x = (double)i - (double)radius;
        kernel[i] = std::exp(-x * x / s2);
        sum += kernel[i];
    }
    for (double& k : kernel) k /= sum;
    Img tmp(w * h), out(w * h);
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) {
            float acc = 0.0f;
            for (size_t ki = 0; ki < kernel.size(); ++ki) {
                const size_t s = x + ki;
                const size_t xx = std::min(s >= radius ? s - radius : 0, w - 1);
                acc += (float)kernel[ki] * src[y * w + xx];
            }
            tmp[y * w + x] = acc;
        }
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x) {
            float acc = 0.0f;
            for (size_t ki = 0; ki < kernel.size(); ++ki) {
                const size_t s = y + ki;
                const size_t yy = std::min(s >= radius ? s - radius : 0, h - 1);
                acc += (float)kernel[ki] * tmp[yy * w + x];
            }
            out[y * w + x] = acc;
        }
    return out;
}

// sift.rs:95-110
Img downsample2(const Img& src, size_t w, size_t h, size_t& nw, size_t& nh) {
    nw = std::max<size_t>(w / 2, 1);
    nh = std::max<size_t>(h / 2, 1);
    Img out(nw * nh);
    for (size_t y = 0; y < nh; ++y)
        for (size_t x = 0; x < nw; ++x) {
            const size_t x0 = std::min(2 * x, w - 1), y0 = std::min(2 * y, h - 1);
            const size_t x1 = std::min(x0 + 1, w - 1), y1 = std::min(y0 + 1, h - 1);
            const float s = src[y0 * w + x0] + src[y0 * w + x1] + src[y1 * w + x0] + src[y1 * w + x1];
            out[y * nw + x] = 0.25f * s;
        }
    return out;
}

struct Octave {
    size_t w, h;
    std::vector<Img> levels, dogs;
};

// 2^((l / NSPO) as i32): the reference truncates the exponent
double level_sigma(int l) { return SIGMA0 * std::pow(2.0, (int)((double)l / (double)NSPO)); }

// sift.rs:112-134
Octave build_octave(Img base, size_t w, size_t h, double first_sigma) {
    Octave o{w, h, {}, {}};
    o.levels.push_back(first_sigma > 1e-4 ? gauss_blur(base, w, h, first_sigma) : std::move(base));
    for (int l = 1; l < NSPO + 3; ++l) {
        const double sp = level_sigma(l - 1), sc = level_sigma(l);
        const double inc = std::sqrt(std::max(sc * sc - sp * sp, 1e-4));
        o.levels.push_back(gauss_blur(o.levels.back(), w, h, inc));
    }
    for (int i = 0; i < NSPO + 2; ++i) {
        Img d(w * h);
        for (size_t p = 0; p < w * h; ++p) d[p] = o.levels[i + 1][p] - o.levels[i][p];
        o.dogs.push_back(std::move(d));
    }
    return o;
}

// sift.rs:137-149
void gradients(const Img& img, size_t w, size_t h, Img& gx, Img& gy) {
    gx.assign(w * h, 0.0f);
    gy.assign(w * h, 0.0f);
    for (size_t y = 1; y + 1 < h; ++y)
        for (size_t x = 1; x + 1 < w; ++x) {
            const size_t i = y * w + x;
            gx[i] = img[i + 1] - img[i - 1];
            gy[i] = img[i + w] - img[i - w];
        }
}

// sift.rs:151-166
float bilinear(const Img& img, size_t w, size_t h, double x, double y) {
    const int64_t x0 = (int64_t)std::floor(x), y0 = (int64_t)std::floor(y);
    const float fx = (float)(x - (double)x0), fy = (float)(y - (double)y0);
    auto cl = [](int64_t v, int64_t m) { return (size_t)std::min(std::max(v, (int64_t)0), m); };
    const int64_t xm = (int64_t)w - 1, ym = (int64_t)h - 1;
    const size_t ax = cl(x0, xm), ay = cl(y0, ym), bx = cl(x0 + 1, xm), by = cl(y0 + 1, ym);
    const float a = img[ay * w + ax] * (1.0f - fx) + img[ay * w + bx] * fx;
    const float b = img[by * w + ax] * (1.0f - fx) + img[by * w + bx] * fx;
    return a * (1.0f - fy) + b * fy;
}

struct RawKp {
    double x, y;
    int octave, level;
    double sigma, response;
};

// nalgebra 0.32 Matrix3::try_inverse (cofactors, each entry divided by the
// determinant); false when the determinant is zero.
bool inverse3(const double m[9], double o[9]) {
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

// sift.rs:176-262
void detect_extrema(const Octave& oc, int octave, double thr, std::vector<RawKp>& out) {
    const size_t w = oc.w, h = oc.h;
    const double edge_lim = (EDGE_THR + 1.0) * (EDGE_THR + 1.0) / EDGE_THR;
    if (w < 3 || h < 3) return;
    for (int level = 1; level <= NSPO; ++level) {
        const Img& dog = oc.dogs[level];
        const Img& below = oc.dogs[level - 1];
        const Img& above = oc.dogs[level + 1];
        for (size_t y = 1; y + 1 < h; ++y)
            for (size_t x = 1; x + 1 < w; ++x) {
                const size_t i = y * w + x;
                const float v = dog[i];
                if ((double)std::fabs(v) < thr) continue;
                bool is_max = true, is_min = true;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dy == 0 && dx == 0) continue;
                        const size_t j = (size_t)((int64_t)y + dy) * w + (size_t)((int64_t)x + dx);
                        for (const Img* im : {&dog, &below, &above}) {
                            const float nb = (*im)[j];
                            if (nb >= v) is_max = false;
                            if (nb <= v) is_min = false;
                        }
                    }
                if (!is_max && !is_min) continue;
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
                if (!inverse3(hm, hi)) continue;
                const double g[3] = {-(double)fdx, -(double)fdy, -(double)fds};
                double off[3];
                for (int r = 0; r < 3; ++r) off[r] = hi[3 * r] * g[0] + hi[3 * r + 1] * g[1] + hi[3 * r + 2] * g[2];
                if (std::fabs(off[0]) > 1.0 || std::fabs(off[1]) > 1.0 || std::fabs(off[2]) > 1.0) continue;
                const double contrast =
                    (double)v + 0.5 * ((double)fdx * off[0] + (double)fdy * off[1] + (double)fds * off[2]);
                if (std::fabs(contrast) < thr) continue;
                const double tr = (double)(dxx + dyy);
                const double det = (double)(dxx * dyy - dxy * dxy);
                if (det <= 0.0 || tr * tr / det > edge_lim) continue;
                out.push_back(RawKp{(double)x + off[0], (double)y + off[1], octave, level, level_sigma(level),
                                    std::fabs(contrast)});
            }
    }
}

double rem_euclid(double a, double b) {
    const double r = std::fmod(a, b);
    return r < 0.0 ? r + std::fabs(b) : r;
}

// sift.rs:274-334
std::vector<double> orientations(const Img& gx, const Img& gy, size_t w, size_t h, double x, double y,
                                 double sigma) {
    double hist[36] = {0};
    const int64_t radius = (int64_t)std::max(std::ceil(3.0 * sigma), 1.0);
    const double s2 = 2.0 * sigma * sigma;
    const int64_t x0 = (int64_t)std::round(x), y0 = (int64_t)std::round(y);
    for (int64_t dy = -radius; dy <= radius; ++dy)
        for (int64_t dx = -radius; dx <= radius; ++dx) {
            const int64_t sx = x0 + dx, sy = y0 + dy;
            if (sx < 1 || sy < 1 || sx >= (int64_t)w - 1 || sy >= (int64_t)h - 1) continue;
            const size_t i = (size_t)sy * w + (size_t)sx;
            const double mag = std::sqrt((double)(gx[i] * gx[i] + gy[i] * gy[i]));
            const double ang = std::atan2((double)gy[i], (double)gx[i]);
            const double wgt = std::exp((-((double)dx * (double)dx) - (double)dy * (double)dy) / s2);
            const double fb = std::floor((ang + PI) / (2.0 * PI) * 36.0);
            size_t bin = !(fb > 0.0) ? 0 : (size_t)fb;  // `as usize`: saturating, NaN -> 0
            bin %= 36;
            hist[bin] += wgt * mag;
        }
    for (int it = 0; it < 2; ++it) {
        double sm[36];
        for (int b = 0; b < 36; ++b) sm[b] = (hist[(b + 35) % 36] + 2.0 * hist[b] + hist[(b + 1) % 36]) / 4.0;
        std::memcpy(hist, sm, sizeof(hist));
    }
    double maxv = 0.0;
    for (double v : hist) maxv = std::fmax(maxv, v);
    if (maxv < 1e-12) return {0.0};
    const double thresh = 0.8 * maxv;
    std::vector<double> peaks;
    for (int b = 0; b < 36; ++b) {
        const double prev = hist[(b + 35) % 36], next = hist[(b + 1) % 36];
        if (hist[b] > prev && hist[b] > next && hist[b] >= thresh) {
            const double denom = hist[b] * 2.0 - prev - next;
            const double d = std::fabs(denom) > 1e-12 ? 0.5 * (prev - next) / denom : 0.0;
            const double theta = ((double)b + d) / 36.0 * 2.0 * PI - PI;
            peaks.push_back(rem_euclid(theta, 2.0 * PI));
            if (peaks.size() >= 4) break;
        }
    }
    if (peaks.empty()) peaks.push_back(0.0);
    return peaks;
}

// sift.rs:340-431
bool descriptor(const Img& gxi, const Img& gyi, size_t w, size_t h, double x, double y, double sigma, double theta,
                float* d) {
    constexpr int D = 4, N = 8;
    const double cell = 3.0 * sigma;
    const int64_t radius = (int64_t)std::ceil(std::sqrt(1.5) * cell * ((double)D + 1.0) * 0.5);
    const double cos_t = std::cos(theta), sin_t = std::sin(theta);
    const double exp_scale = -1.0 / ((double)(D * D) * 0.5);
    double hist[D * D][N] = {{0}};
    const double half = (double)D * 0.5;
    for (int64_t dy = -radius; dy <= radius; ++dy)
        for (int64_t dx = -radius; dx <= radius; ++dx) {
            const double sx = x + (double)dx, sy = y + (double)dy;
            if (sx < 1.0 || sy < 1.0 || sx >= (double)w - 2.0 || sy >= (double)h - 2.0) continue;
            const double gx = (double)bilinear(gxi, w, h, sx, sy);
            const double gy = (double)bilinear(gyi, w, h, sx, sy);
            const double mag = std::sqrt(gx * gx + gy * gy);
            if (mag < 1e-12) continue;
            const double rx = cos_t * (double)dx + sin_t * (double)dy;
            const double ry = -sin_t * (double)dx + cos_t * (double)dy;
            const double bx = rx / cell + half - 0.5;
            const double by = ry / cell + half - 0.5;
            if (bx < -1.0 || by < -1.0 || bx > (double)D || by > (double)D) continue;
            const double ang = std::atan2(gy, gx) - theta;
            const double ob = rem_euclid(ang, 2.0 * PI) / (2.0 * PI) * (double)N;
            double wgt = ((bx - half + 0.5) * (bx - half + 0.5) + (by - half + 0.5) * (by - half + 0.5)) * exp_scale;
            wgt = std::exp(wgt) * mag;
            const int64_t bx0 = (int64_t)std::floor(bx), by0 = (int64_t)std::floor(by), ob0 = (int64_t)std::floor(ob);
            const double fx = bx - (double)bx0, fy = by - (double)by0, fo = ob - (double)ob0;
            for (int iy = 0; iy < 2; ++iy)
                for (int ix = 0; ix < 2; ++ix) {
                    const int64_t bxi = bx0 + ix, byi = by0 + iy;
                    if (bxi < 0 || byi < 0 || bxi >= D || byi >= D) continue;
                    const double wy = iy == 0 ? 1.0 - fy : fy;
                    const double wx = ix == 0 ? 1.0 - fx : fx;
                    for (int io = 0; io < 2; ++io) {
                        const int64_t obi = ((ob0 + io) % N + N) % N;
                        const double wo = io == 0 ? 1.0 - fo : fo;
                        hist[byi * D + bxi][obi] += wgt * wx * wy * wo;
                    }
                }
        }
    for (int k = 0; k < D * D; ++k)
        for (int b = 0; b < N; ++b) d[k * N + b] = (float)hist[k][b];
    float ss = 0.0f;
    for (int i = 0; i < DESC_LEN; ++i) ss += d[i] * d[i];
    const float norm = std::sqrt(ss);
    if (norm < 1e-6f) return false;
    for (int i = 0; i < DESC_LEN; ++i) d[i] /= norm;
    for (int i = 0; i < DESC_LEN; ++i)
        if (d[i] > 0.2f) d[i] = 0.2f;
    float ss2 = 0.0f;
    for (int i = 0; i < DESC_LEN; ++i) ss2 += d[i] * d[i];
    const float norm2 = std::sqrt(ss2);
    if (norm2 < 1e-6f) return false;
    for (int i = 0; i < DESC_LEN; ++i) d[i] /= norm2;
    return true;
}

struct OutKp {
    double resp, x, y;
    float d[DESC_LEN];
};

}  // namespace

extern "C" {

int orc_extract_sift(const uint8_t* gray, const uint8_t* rgb, int32_t w32, int32_t h32, uint32_t max_features,
                     double contrast_thr, double** pts_out, float** desc_out, uint8_t** colors_out,
                     uint64_t* n_out, uint64_t* n_raw_out) {
    if (!gray || !rgb || w32 <= 0 || h32 <= 0 || !pts_out || !desc_out || !colors_out || !n_out) return -1;
    const size_t w = (size_t)w32, h = (size_t)h32;
    Img base(w * h);
    for (size_t i = 0; i < w * h; ++i) base[i] = (float)gray[i] / 255.0f;
    size_t n_oct = 1;
    while ((std::max(w, h) >> n_oct) >= 40 && n_oct < 8) ++n_oct;
    std::vector<RawKp> raw;
    std::vector<Octave> octaves;
    Img ob = base;
    size_t ow = w, oh = h;
    for (size_t o = 0; o < n_oct; ++o) {
        const double fs =
            o == 0 ? std::sqrt(std::max(SIGMA0 * SIGMA0 - ASSUMED_BLUR * ASSUMED_BLUR, 1e-4)) : 0.0;
        Octave oc = build_octave(ob, ow, oh, fs);
        detect_extrema(oc, (int)o, contrast_thr, raw);
        size_t nw, nh;
        Img next = downsample2(oc.levels[NSPO], ow, oh, nw, nh);
        octaves.push_back(std::move(oc));
        ob = std::move(next);
        ow = nw;
        oh = nh;
    }
    if (n_raw_out) *n_raw_out = raw.size();
    std::vector<OutKp> outs;
    for (size_t o = 0; o < octaves.size(); ++o) {
        const Octave& oc = octaves[o];
        const double scale = std::pow(2.0, (int)o);
        Img gx[NSPO + 2], gy[NSPO + 2];
        bool have[NSPO + 2] = {false};
        for (const RawKp& kp : raw) {
            if (kp.octave != (int)o) continue;
            const int li = kp.level;
            if (!have[li]) {
                gradients(oc.levels[li], oc.w, oc.h, gx[li], gy[li]);
                have[li] = true;
            }
            const double x0 = kp.x * scale, y0 = kp.y * scale;
            if (x0 < 8.0 || y0 < 8.0 || x0 >= (double)w - 8.0 || y0 >= (double)h - 8.0) continue;
            for (double theta : orientations(gx[li], gy[li], oc.w, oc.h, kp.x, kp.y, 1.5 * kp.sigma)) {
                OutKp k;
                if (descriptor(gx[li], gy[li], oc.w, oc.h, kp.x, kp.y, kp.sigma, theta, k.d)) {
                    k.resp = kp.response;
                    k.x = x0;
                    k.y = y0;
                    outs.push_back(k);
                }
            }
        }
    }
    std::stable_sort(outs.begin(), outs.end(), [](const OutKp& a, const OutKp& b) { return b.resp < a.resp; });
    if (outs.size() > max_features) outs.resize(max_features);
    const size_t n = outs.size();
    double* pts = (double*)std::malloc(sizeof(double) * 2 * std::max<size_t>(n, 1));
    float* desc = (float*)std::malloc(sizeof(float) * DESC_LEN * std::max<size_t>(n, 1));
    uint8_t* col = (uint8_t*)std::malloc(3 * std::max<size_t>(n, 1));
    if (!pts || !desc || !col) {
        std::free(pts);
        std::free(desc);
        std::free(col);
        return -3;
    }
    for (size_t k = 0; k < n; ++k) {
        const double x = std::min(std::max(outs[k].x, 0.0), (double)(w - 1));
        const double y = std::min(std::max(outs[k].y, 0.0), (double)(h - 1));
        const size_t px = std::min((size_t)std::round(x), w - 1), py = std::min((size_t)std::round(y), h - 1);
        pts[2 * k] = x;
        pts[2 * k + 1] = y;
        std::memcpy(desc + DESC_LEN * k, outs[k].d, sizeof(float) * DESC_LEN);
        for (int c = 0; c < 3; ++c) col[3 * k + c] = rgb[3 * (py * w + px) + c];
    }
    *pts_out = pts;
    *desc_out = desc;
    *colors_out = col;
    *n_out = n;
    return 0;
}

}  // extern "C"

extern "C" {

// sfm-lite/src/matching.rs:22-95  match_pair: nearest and second-nearest
// neighbour by serial f32 squared distance in both directions, Lowe ratio
// test both ways and the mutual check.  out_a / out_b need min(na, nb)
// entries.
void orc_match_pair(const float* a, uint32_t na, const float* b, uint32_t nb, double ratio64, uint32_t* out_a,
                    uint32_t* out_b, uint64_t* n_out) {
    *n_out = 0;
    if (na == 0 || nb == 0) return;
    struct Best {
        uint32_t idx;
        float d1, d2;
    };
    auto scan = [](const float* q, const float* set, uint32_t n) {
        float best = INFINITY, second = INFINITY;
        uint32_t bi = UINT32_MAX;
        for (uint32_t j = 0; j < n; ++j) {
            float s = 0.0f;
            for (int k = 0; k < DESC_LEN; ++k) {
                const float d = q[k] - set[(size_t)j * DESC_LEN + k];
                s += d * d;
            }
            if (s < best) {
                second = best;
                best = s;
                bi = j;
            } else if (s < second) {
                second = s;
            }
        }
        return Best{bi, best, second};
    };
    std::vector<Best> fwd(na), bwd(nb);
    for (uint32_t i = 0; i < na; ++i) fwd[i] = scan(a + (size_t)i * DESC_LEN, b, nb);
    // backward distances subtract in the same order (a - b), as the reference
    for (uint32_t j = 0; j < nb; ++j) {
        float best = INFINITY, second = INFINITY;
        uint32_t bi = UINT32_MAX;
        for (uint32_t i = 0; i < na; ++i) {
            float s = 0.0f;
            for (int k = 0; k < DESC_LEN; ++k) {
                const float d = a[(size_t)i * DESC_LEN + k] - b[(size_t)j * DESC_LEN + k];
                s += d * d;
            }
            if (s < best) {
                second = best;
                best = s;
                bi = i;
            } else if (s < second) {
                second = s;
            }
        }
        bwd[j] = Best{bi, best, second};
    }
    const float ratio = (float)ratio64;
    uint64_t n = 0;
    for (uint32_t i = 0; i < na; ++i) {
        const Best& f = fwd[i];
        if (f.idx == UINT32_MAX || !std::isfinite(f.d2)) continue;
        if (f.d1 > 0.9f || f.d1 > ratio * f.d2) continue;
        const Best& g = bwd[f.idx];
        if (g.idx != i) continue;
        if (!std::isfinite(g.d2) || g.d1 > ratio * g.d2) continue;
        out_a[n] = i;
        out_b[n] = f.idx;
        ++n;
    }
    *n_out = n;
}

}  // extern "C"
