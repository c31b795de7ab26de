"""A second, independent restatement of sfm-lite's extract_sift
(sfm-lite/src/sift.rs:51-555) in numpy f32/f64 arithmetic and Python's math
module (the host libm, as the C++ oracle and Rust's f64 methods use),
checked against the C++ oracle (oracle/sift_oracle.cpp) on small images.
Two restatements written separately that agree bit for bit pin the oracle
against transcription mistakes; neither is pinned to the Rust reference,
which cannot be built here."""
import math

import numpy as np
import pytest

from oracle import oracle
from rustcolmap_b200 import scene

F = np.float32
NSPO, SIGMA0, ASSUMED_BLUR, EDGE_THR = 3, 1.6, 0.5, 10.0


def gauss_blur(src, sigma):
    """sift.rs:51-93: f64 weights cast to f32, clamped taps summed in order."""
    if sigma < 1e-4:
        return src.copy()
    radius = int(max(math.ceil(sigma * 3.0), 1.0))
    s2 = 2.0 * sigma * sigma
    k = [math.exp(-(float(i - radius) * float(i - radius)) / s2) for i in range(2 * radius + 1)]
    tot = 0.0
    for v in k:
        tot += v
    k = [F(v / tot) for v in k]
    h, w = src.shape
    xs = np.arange(w)
    tmp = np.zeros_like(src)
    for ki, kv in enumerate(k):
        idx = np.minimum(np.maximum(xs + ki - radius, 0), w - 1)
        tmp = tmp + kv * src[:, idx]
    ys = np.arange(h)
    out = np.zeros_like(src)
    for ki, kv in enumerate(k):
        idx = np.minimum(np.maximum(ys + ki - radius, 0), h - 1)
        out = out + kv * tmp[idx, :]
    return out


def level_sigma(l):
    return SIGMA0 * 2.0 ** int(l / NSPO)


def build_octave(base, first_sigma):
    levels = [gauss_blur(base, first_sigma) if first_sigma > 1e-4 else base]
    for l in range(1, NSPO + 3):
        sp, sc = level_sigma(l - 1), level_sigma(l)
        levels.append(gauss_blur(levels[-1], math.sqrt(max(sc * sc - sp * sp, 1e-4))))
    dogs = [levels[i + 1] - levels[i] for i in range(NSPO + 2)]
    return levels, dogs


def downsample2(src):
    h, w = src.shape
    nw, nh = max(w // 2, 1), max(h // 2, 1)
    x0 = np.minimum(2 * np.arange(nw), w - 1)
    y0 = np.minimum(2 * np.arange(nh), h - 1)
    x1, y1 = np.minimum(x0 + 1, w - 1), np.minimum(y0 + 1, h - 1)
    s = src[np.ix_(y0, x0)] + src[np.ix_(y0, x1)] + src[np.ix_(y1, x0)] + src[np.ix_(y1, x1)]
    return F(0.25) * s


def inv3(m):
    """nalgebra 0.32 Matrix3::try_inverse (cofactors / determinant)."""
    (m11, m12, m13), (m21, m22, m23), (m31, m32, m33) = m
    a = m22 * m33 - m32 * m23
    b = m21 * m33 - m31 * m23
    c = m21 * m32 - m31 * m22
    det = m11 * a - m12 * b + m13 * c
    if det == 0.0:
        return None
    return [[a / det, (m13 * m32 - m33 * m12) / det, (m12 * m23 - m22 * m13) / det],
            [-b / det, (m11 * m33 - m31 * m13) / det, (m13 * m21 - m23 * m11) / det],
            [c / det, (m12 * m31 - m32 * m11) / det, (m11 * m22 - m21 * m12) / det]]


def detect(dogs, octave, thr, out):
    """sift.rs:176-262 (python floats are f64; F() keeps the f32 steps)."""
    h, w = dogs[0].shape
    edge_lim = (EDGE_THR + 1.0) ** 2 / EDGE_THR
    for level in range(1, NSPO + 1):
        d, lo, hi = dogs[level], dogs[level - 1], dogs[level + 1]
        for y in range(1, h - 1):
            for x in range(1, w - 1):
                v = d[y, x]
                if float(abs(v)) < thr:
                    continue
                nb = np.concatenate([d[y - 1:y + 2, x - 1:x + 2].ravel(), lo[y - 1:y + 2, x - 1:x + 2].ravel(),
                                     hi[y - 1:y + 2, x - 1:x + 2].ravel()])
                nb = np.delete(nb, [4, 13, 22])  # the centre of every level is skipped
                is_max, is_min = bool((nb < v).all()), bool((nb > v).all())
                if not (is_max or is_min):
                    continue
                dx = F(0.5) * (d[y, x + 1] - d[y, x - 1])
                dy = F(0.5) * (d[y + 1, x] - d[y - 1, x])
                ds = F(0.5) * (hi[y, x] - lo[y, x])
                dxx = d[y, x + 1] + d[y, x - 1] - F(2.0) * v
                dyy = d[y + 1, x] + d[y - 1, x] - F(2.0) * v
                dss = hi[y, x] + lo[y, x] - F(2.0) * v
                dxy = F(0.25) * (d[y + 1, x + 1] + d[y - 1, x - 1] - d[y + 1, x - 1] - d[y - 1, x + 1])
                dxs = F(0.25) * (hi[y, x + 1] + lo[y, x - 1] - hi[y, x - 1] - lo[y, x + 1])
                dys = F(0.25) * (hi[y + 1, x] + lo[y - 1, x] - hi[y - 1, x] - lo[y + 1, x])
                m = [[float(dxx), float(dxy), float(dxs)], [float(dxy), float(dyy), float(dys)],
                     [float(dxs), float(dys), float(dss)]]
                hinv = inv3(m)
                if hinv is None:
                    continue
                g = [-float(dx), -float(dy), -float(ds)]
                off = [r[0] * g[0] + r[1] * g[1] + r[2] * g[2] for r in hinv]
                if abs(off[0]) > 1.0 or abs(off[1]) > 1.0 or abs(off[2]) > 1.0:
                    continue
                contrast = float(v) + 0.5 * (float(dx) * off[0] + float(dy) * off[1] + float(ds) * off[2])
                if abs(contrast) < thr:
                    continue
                tr = float(dxx + dyy)
                det = float(dxx * dyy - dxy * dxy)
                if det <= 0.0 or tr * tr / det > edge_lim:
                    continue
                out.append((x + off[0], y + off[1], octave, level, level_sigma(level), abs(contrast)))


def gradients(img):
    gx = np.zeros_like(img)
    gy = np.zeros_like(img)
    gx[1:-1, 1:-1] = img[1:-1, 2:] - img[1:-1, :-2]
    gy[1:-1, 1:-1] = img[2:, 1:-1] - img[:-2, 1:-1]
    return gx, gy


def rem_euclid(a, b):
    r = math.fmod(a, b)
    return r + abs(b) if r < 0.0 else r


def orientations(gx, gy, x, y, sigma):
    """sift.rs:274-334."""
    h, w = gx.shape
    hist = [0.0] * 36
    radius = int(max(math.ceil(3.0 * sigma), 1.0))
    s2 = 2.0 * sigma * sigma
    def rnd(v):  # f64::round (half away from zero) for v >= 0, without the x + 0.5 rounding trap
        f = math.floor(v)
        return int(f) + (1 if v - f >= 0.5 else 0)
    x0, y0 = rnd(x), rnd(y)
    for dy in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            sx, sy = x0 + dx, y0 + dy
            if sx < 1 or sy < 1 or sx >= w - 1 or sy >= h - 1:
                continue
            a, b = gx[sy, sx], gy[sy, sx]
            mag = math.sqrt(float(a * a + b * b))
            ang = math.atan2(float(b), float(a))
            wgt = math.exp((-(float(dx) ** 2) - float(dy) ** 2) / s2)
            fb = math.floor((ang + math.pi) / (2.0 * math.pi) * 36.0)
            hist[(int(fb) if fb > 0 else 0) % 36] += wgt * mag
    for _ in range(2):
        hist = [(hist[(b + 35) % 36] + 2.0 * hist[b] + hist[(b + 1) % 36]) / 4.0 for b in range(36)]
    maxv = 0.0
    for v in hist:
        maxv = max(maxv, v)
    if maxv < 1e-12:
        return [0.0]
    peaks = []
    for b in range(36):
        prev, nxt = hist[(b + 35) % 36], hist[(b + 1) % 36]
        if hist[b] > prev and hist[b] > nxt and hist[b] >= 0.8 * maxv:
            denom = hist[b] * 2.0 - prev - nxt
            d = 0.5 * (prev - nxt) / denom if abs(denom) > 1e-12 else 0.0
            peaks.append(rem_euclid((b + d) / 36.0 * 2.0 * math.pi - math.pi, 2.0 * math.pi))
            if len(peaks) >= 4:
                break
    return peaks or [0.0]


def bilinear(img, x, y):
    h, w = img.shape
    x0, y0 = int(math.floor(x)), int(math.floor(y))
    fx, fy = F(x - x0), F(y - y0)
    cx = lambda v: min(max(v, 0), w - 1)
    cy = lambda v: min(max(v, 0), h - 1)
    a = img[cy(y0), cx(x0)] * (F(1) - fx) + img[cy(y0), cx(x0 + 1)] * fx
    b = img[cy(y0 + 1), cx(x0)] * (F(1) - fx) + img[cy(y0 + 1), cx(x0 + 1)] * fx
    return a * (F(1) - fy) + b * fy


def descriptor(gx, gy, x, y, sigma, theta):
    """sift.rs:340-431."""
    h, w = gx.shape
    D, N = 4, 8
    cell = 3.0 * sigma
    radius = int(math.ceil(math.sqrt(1.5) * cell * (D + 1.0) * 0.5))
    ct, st = math.cos(theta), math.sin(theta)
    exp_scale = -1.0 / (D * D * 0.5)
    hist = [[0.0] * N for _ in range(D * D)]
    half = D * 0.5
    for dy in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            sx, sy = x + dx, y + dy
            if sx < 1.0 or sy < 1.0 or sx >= w - 2.0 or sy >= h - 2.0:
                continue
            gxv, gyv = float(bilinear(gx, sx, sy)), float(bilinear(gy, sx, sy))
            mag = math.sqrt(gxv * gxv + gyv * gyv)
            if mag < 1e-12:
                continue
            rx = ct * dx + st * dy
            ry = -st * dx + ct * dy
            bx, by = rx / cell + half - 0.5, ry / cell + half - 0.5
            if bx < -1.0 or by < -1.0 or bx > D or by > D:
                continue
            ob = rem_euclid(math.atan2(gyv, gxv) - theta, 2.0 * math.pi) / (2.0 * math.pi) * N
            wgt = math.exp(((bx - half + 0.5) * (bx - half + 0.5) + (by - half + 0.5) * (by - half + 0.5))
                           * exp_scale) * mag
            bx0, by0, ob0 = math.floor(bx), math.floor(by), math.floor(ob)
            fx, fy, fo = bx - bx0, by - by0, ob - ob0
            for iy in range(2):
                for ix in range(2):
                    bxi, byi = bx0 + ix, by0 + iy
                    if bxi < 0 or byi < 0 or bxi >= D or byi >= D:
                        continue
                    wy, wx = (1.0 - fy) if iy == 0 else fy, (1.0 - fx) if ix == 0 else fx
                    for io in range(2):
                        wo = (1.0 - fo) if io == 0 else fo
                        hist[byi * D + bxi][(ob0 + io) % N] += wgt * wx * wy * wo
    d = np.array([F(v) for row in hist for v in row], np.float32)
    ss = F(0)
    for v in d:
        ss = ss + v * v
    norm = np.sqrt(ss)  # f32 sqrt, correctly rounded
    if norm < F(1e-6):
        return None
    d = d / norm
    d = np.where(d > F(0.2), F(0.2), d).astype(np.float32)
    ss = F(0)
    for v in d:
        ss = ss + v * v
    norm2 = np.sqrt(ss)
    if norm2 < F(1e-6):
        return None
    return (d / norm2).astype(np.float32)


def extract(gray, rgb, max_features=2048, thr=0.0067):
    """sift.rs:435-555 on an image at working resolution."""
    h, w = gray.shape
    base = gray.astype(np.float32) / F(255.0)
    n_oct = 1
    while (max(w, h) >> n_oct) >= 40 and n_oct < 8:
        n_oct += 1
    raw, octaves = [], []
    ob = base
    for o in range(n_oct):
        fs = math.sqrt(max(SIGMA0 * SIGMA0 - ASSUMED_BLUR * ASSUMED_BLUR, 1e-4)) if o == 0 else 0.0
        levels, dogs = build_octave(ob, fs)
        if min(ob.shape) >= 3:
            detect(dogs, o, thr, raw)
        octaves.append(levels)
        ob = downsample2(levels[NSPO])
    outs = []
    for o, levels in enumerate(octaves):
        scale = 2.0 ** o
        grads = {}
        for (x, y, ko, level, sigma, resp) in raw:
            if ko != o:
                continue
            if level not in grads:
                grads[level] = gradients(levels[level])
            gx, gy = grads[level]
            x0, y0 = x * scale, y * scale
            if x0 < 8.0 or y0 < 8.0 or x0 >= w - 8.0 or y0 >= h - 8.0:
                continue
            for th in orientations(gx, gy, x, y, 1.5 * sigma):
                d = descriptor(gx, gy, x, y, sigma, th)
                if d is not None:
                    outs.append((resp, x0, y0, d))
    outs = sorted(outs, key=lambda t: -t[0])[:max_features]  # stable
    pts = np.array([[min(max(x, 0.0), w - 1.0), min(max(y, 0.0), h - 1.0)] for _, x, y, _ in outs]).reshape(-1, 2)
    desc = np.array([d for *_, d in outs], np.float32).reshape(-1, 128)
    px = np.minimum(np.floor(pts + 0.5).astype(int), [w - 1, h - 1]) if len(pts) else np.zeros((0, 2), int)
    col = rgb[px[:, 1], px[:, 0]] if len(pts) else np.zeros((0, 3), np.uint8)
    return pts, desc, col, len(raw)


@pytest.mark.parametrize("which", ["blob", "view", "view3"])
def test_numpy_restatement_equals_oracle(which):
    if which == "view3":  # 160x120: three octaves, keypoints scaled by 2 and 4
        v = scene.corner_room(seed=8, n_views=2, w=160, h=120, f=180.0, arc_deg=20.0, n_patches=40,
                              per_view_sparse=10).views[0]
        g, rgb = np.ascontiguousarray(v.gray), np.ascontiguousarray(v.rgb)
    elif which == "blob":
        yy, xx = np.mgrid[0:72, 0:96]
        g = (30 + 200 * np.exp(-((xx - 47.5) ** 2 + (yy - 35.0) ** 2) / 50.0)
             + 40 * np.exp(-((xx - 20.0) ** 2 + (yy - 50.0) ** 2) / 8.0)).astype(np.uint8)
        rgb = np.repeat(g[:, :, None], 3, axis=2)
    else:
        v = scene.corner_room(seed=3, n_views=2, w=96, h=72, f=110.0, arc_deg=20.0, n_patches=30,
                              per_view_sparse=10).views[0]
        g, rgb = np.ascontiguousarray(v.gray), np.ascontiguousarray(v.rgb)
    pts, desc, col, nraw = extract(g, rgb)
    opts_, odesc, ocol, onraw = oracle.extract_sift(g, rgb)
    assert nraw == onraw and len(pts) > 0
    assert np.array_equal(pts, opts_) and np.array_equal(col, ocol)
    assert np.array_equal(desc.view(np.uint32), odesc.view(np.uint32))
