"""Generates tests/golden/*.npz: golden vectors for the dense-MVS path.

The reference (Rust) cannot be built or run where this project is developed
and ships no golden vectors, so these fixtures come from a second,
independent restatement of the reference written here in pure Python with
numpy float32/float64 scalars (IEEE, one rounding per operation, like Rust).
They pin the C++ oracle against a transcription error; they do not pin either
restatement against the reference binary ("parity unpinned").

Each function cites the reference lines it restates.  Inputs are tiny images
rendered by the project's scene generator and stored in the fixture, so the
fixture is self-contained.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

F = np.float32
M64 = (1 << 64) - 1


# ---------------------------------------------------------------- census
def census_map(gray):
    """mvs/src/lib.rs:119-142 on gray = u8/255 (f32)."""
    h, w = gray.shape
    g = gray.astype(np.float32) / F(255.0)
    out = np.zeros((h, w), np.uint64)
    for y in range(h):
        for x in range(w):
            c = g[y, x]
            bits = 0
            for dy in range(-3, 4):
                for dx in range(-3, 4):
                    if dx == 0 and dy == 0:
                        continue
                    xx = min(max(x + dx, 0), w - 1)
                    yy = min(max(y + dy, 0), h - 1)
                    if g[yy, xx] < c:
                        bits |= 1 << ((dy + 3) * 7 + (dx + 3))
            out[y, x] = bits
    return out


# ---------------------------------------------------------------- rng
def pixel_rng(x, y, salt):
    """mvs/src/stereo.rs:47-57 (wrapping u64)."""
    s = ((x * 0x9E3779B97F4A7C15) & M64) ^ ((y * 0xC2B2AE3D27D4EB4F) & M64) ^ ((salt * 0x165667B19E3779F9) & M64)
    s ^= s >> 30
    s = (s * 0xBF58476D1CE4E5B9) & M64
    s ^= s >> 27
    s = (s * 0x94D049BB133111EB) & M64
    return s ^ (s >> 31)


class Rng:
    def __init__(self, seed):
        self.s = seed

    def next_u64(self):
        """stereo.rs:59-67"""
        x = self.s
        x ^= (x << 13) & M64
        x ^= x >> 7
        x ^= (x << 17) & M64
        self.s = x
        return x

    def uniform(self):
        """stereo.rs:69-72"""
        return F(self.next_u64() >> 40) / F(1 << 24)

    def gauss(self):
        """stereo.rs:74-78"""
        a = self.uniform()
        b = self.uniform()
        c = self.uniform()
        return a + b + c - F(1.5)


def f32_as_i32(v):
    """Rust `f32 as i32`."""
    if np.isnan(v):
        return 0
    if v >= F(2147483648.0):
        return 2147483647
    if v < F(-2147483648.0):
        return -2147483648
    return int(v)  # truncation toward zero


# ---------------------------------------------------------------- geometry
def cam_normalize(cam, u, v):
    """sfm-lite/src/geom.rs:28-42 (f64)."""
    f, cx, cy, k = (float(c) for c in cam)
    xn = (u - cx) / f
    yn = (v - cy) / f
    for _ in range(2):
        r2 = xn * xn + yn * yn
        d = 1.0 + k * r2
        if abs(d) < 1e-12:
            break
        xn = (u - cx) / (f * d)
        yn = (v - cy) / (f * d)
    return xn, yn


class Workspace:
    """mvs/src/stereo.rs:103-151"""

    def __init__(self, views, census, ref, srcs, zmin, zmax):
        r = views[ref]
        self.w, self.h = r["w"], r["h"]
        self.census = census[ref]
        self.rx = np.zeros((self.h, self.w), np.float32)
        self.ry = np.zeros((self.h, self.w), np.float32)
        for y in range(self.h):
            for x in range(self.w):
                a, b = cam_normalize(r["cam"], float(x), float(y))
                self.rx[y, x] = F(a)
                self.ry[y, x] = F(b)
        self.src = []
        Rr, tr = r["R"], r["t"]
        for s in srcs:
            sv = views[s]
            Rs, ts = sv["R"], sv["t"]
            rs64 = [[Rs[i][0] * Rr[j][0] + Rs[i][1] * Rr[j][1] + Rs[i][2] * Rr[j][2] for j in range(3)]
                    for i in range(3)]
            ts64 = [ts[i] - (rs64[i][0] * tr[0] + rs64[i][1] * tr[1] + rs64[i][2] * tr[2]) for i in range(3)]
            self.src.append(dict(census=census[s], w=sv["w"], h=sv["h"], f=F(sv["cam"][0]), cx=F(sv["cam"][1]),
                                 cy=F(sv["cam"][2]), k=F(sv["cam"][3]),
                                 rs=[F(rs64[i][j]) for i in range(3) for j in range(3)],
                                 ts=[F(x) for x in ts64]))
        self.zmin, self.zmax = F(zmin), F(zmax)


def plane_cost(ws, px, py, nx, ny, nz, d, hint):
    """mvs/src/stereo.rs:158-228; returns (cost, integer hamming sum)."""
    w, h = ws.w, ws.h
    nsrc = F(len(ws.src))
    span = F(5.0)
    total = span * span * nsrc
    s_ = F(0.0)
    hs = 0
    for si, s in enumerate(ws.src):
        rs, ts = s["rs"], s["ts"]
        for dy in range(-2, 3):
            ycl = min(max(py + dy, 0), h - 1)
            for dx in range(-2, 3):
                xcl = min(max(px + dx, 0), w - 1)
                xo, yo = ws.rx[ycl, xcl], ws.ry[ycl, xcl]
                denom = nx * xo + ny * yo + nz
                if denom < F(0.05):
                    s_ = s_ + F(1.0)
                    hs += 48
                    continue
                z = d / denom
                xr = z * xo
                yr = z * yo
                xs = rs[0] * xr + rs[1] * yr + rs[2] * z + ts[0]
                ys = rs[3] * xr + rs[4] * yr + rs[5] * z + ts[1]
                zs = rs[6] * xr + rs[7] * yr + rs[8] * z + ts[2]
                if zs < F(1e-3):
                    s_ = s_ + F(1.0)
                    hs += 48
                    continue
                xn = xs / zs
                yn = ys / zs
                dist = F(1.0) + s["k"] * (xn * xn + yn * yn)
                u = f32_as_i32(s["f"] * xn * dist + s["cx"])
                v = f32_as_i32(s["f"] * yn * dist + s["cy"])
                if u < 0 or v < 0 or u >= s["w"] or v >= s["h"]:
                    s_ = s_ + F(1.0)
                    hs += 48
                    continue
                pc = bin(int(ws.census[ycl, xcl]) ^ int(s["census"][v, u])).count("1")
                hs += pc
                s_ = s_ + F(pc) / F(48.0)
            rows_done = F(dy + 3)
            if s_ / (rows_done * span * F(si + 1)) > hint + F(0.12):
                return F(1e9), hs
    return s_ / total, hs


def estimate_depth(views, census, ref, srcs, zmin, zmax, num_hyp, sweeps, cost_thr):
    """mvs/src/stereo.rs:234-394; returns depth, cost, normals (h, w, 3)."""
    ws = Workspace(views, census, ref, srcs, zmin, zmax)
    w, h = ws.w, ws.h
    inv_min = F(1.0) / ws.zmax
    inv_max = F(1.0) / ws.zmin
    nh = max(num_hyp, 2)
    prev = np.zeros((h, w, 5), np.float32)
    for y in range(h):
        for x in range(w):
            best_c, best_d = F(np.inf), F(0.0)
            for hi in range(nh):
                inv = inv_min + (inv_max - inv_min) * F(hi) / F(nh - 1)
                d = F(1.0) / inv
                c, _ = plane_cost(ws, x, y, F(0.0), F(0.0), F(1.0), d, best_c + F(0.02))
                if c < best_c:
                    best_c, best_d = c, d
            prev[y, x] = (0.0, 0.0, 1.0, best_d, min(best_c, F(1.0)))
    n_passes = max(sweeps, 1) * 2
    zlo, zhi = ws.zmin * F(0.5), ws.zmax * F(2.0)
    for p in range(n_passes):
        t = F(p) / F(n_passes)
        sig_inv = F(0.02) * np.power(F(0.28), t * F(4.0))
        sig_n = F(0.30) * np.power(F(0.42), t * F(4.0))
        nxt = prev.copy()
        for y in range(h):
            for x in range(w):
                rng = Rng(pixel_rng(x, y, p + 7))
                cur = prev[y, x]
                best_c = cur[4]
                bn = [cur[0], cur[1], cur[2]]
                rxi, ryi = ws.rx[y, x], ws.ry[y, x]
                bd = cur[3] * (bn[0] * rxi + bn[1] * ryi + bn[2])
                for dx, dy in ((-1, 0), (1, 0), (0, -1), (0, 1)):
                    xx, yy = x + dx, y + dy
                    if xx < 0 or yy < 0 or xx >= w or yy >= h:
                        continue
                    nb = prev[yy, xx]
                    a_nb = nb[0] * ws.rx[yy, xx] + nb[1] * ws.ry[yy, xx] + nb[2]
                    if a_nb < F(0.1):
                        continue
                    d_plane = nb[3] * a_nb
                    a_here = nb[0] * rxi + nb[1] * ryi + nb[2]
                    if a_here < F(0.1):
                        continue
                    zc = d_plane / a_here
                    if not (zlo <= zc <= zhi):
                        continue
                    c, _ = plane_cost(ws, x, y, nb[0], nb[1], nb[2], d_plane, best_c + F(0.02))
                    if c < best_c:
                        best_c, bn, bd = c, [nb[0], nb[1], nb[2]], d_plane
                for _ in range(3):
                    inv = F(1.0) / max(cur[3], F(1e-6))
                    inv_new = inv + sig_inv * (inv_max - inv_min) * rng.gauss()
                    if inv_new <= F(0.0):
                        continue
                    zc = F(1.0) / inv_new
                    if not (zlo <= zc <= zhi):
                        continue
                    nnx = cur[0] + sig_n * rng.gauss()
                    nny = cur[1] + sig_n * rng.gauss()
                    nnz = cur[2] + sig_n * rng.gauss()
                    ln = np.sqrt(nnx * nnx + nny * nny + nnz * nnz)
                    if ln < F(1e-6):
                        continue
                    nnx, nny, nnz = nnx / ln, nny / ln, nnz / ln
                    a_here = nnx * rxi + nny * ryi + nnz
                    if a_here < F(0.1):
                        continue
                    d_plane = zc * a_here
                    c, _ = plane_cost(ws, x, y, nnx, nny, nnz, d_plane, best_c + F(0.02))
                    if c < best_c:
                        best_c, bn, bd = c, [nnx, nny, nnz], d_plane
                if best_c < cur[4]:
                    a_here = bn[0] * rxi + bn[1] * ryi + bn[2]
                    if a_here > F(0.05):
                        nxt[y, x] = (bn[0], bn[1], bn[2], bd / a_here, min(best_c, F(1.0)))
        prev = nxt
    depth = prev[:, :, 3].copy()
    cost = prev[:, :, 4].copy()
    for y in range(h):
        for x in range(w):
            tex = bin(int(ws.census[y, x])).count("1")
            ok = 4 <= tex <= 44 and cost[y, x] < F(cost_thr) and depth[y, x] > zlo and depth[y, x] < zhi
            if not ok:
                depth[y, x] = F(0.0)
    return depth, cost, prev[:, :, :3].copy()


# ---------------------------------------------------------------- fusion
def _mv(R, x):
    return [R[i][0] * x[0] + R[i][1] * x[1] + R[i][2] * x[2] for i in range(3)]


def _mtv(R, x):
    return [R[0][i] * x[0] + R[1][i] * x[1] + R[2][i] * x[2] for i in range(3)]


def sample_depth(dm, u, v):
    """mvs/src/fuse.rs:32-62"""
    h, w = dm.shape
    u0 = int(np.floor(u))
    v0 = int(np.floor(v))
    if u0 < 0 or v0 < 0 or u0 + 1 >= w or v0 + 1 >= h:
        return 0.0
    fx = F(u - float(u0))
    fy = F(v - float(v0))
    taps = [(dm[v0, u0], (F(1) - fx) * (F(1) - fy)), (dm[v0, u0 + 1], fx * (F(1) - fy)),
            (dm[v0 + 1, u0], (F(1) - fx) * fy), (dm[v0 + 1, u0 + 1], fx * fy)]
    acc, wsum = F(0), F(0)
    for d, wt in taps:
        if d > F(0):
            acc = acc + d * wt
            wsum = wsum + wt
    return float(acc / wsum) if wsum > F(1e-6) else 0.0


def fuse(views, depth_maps, order, sparse, min_consistent, depth_diff, voxel_rel):
    """mvs/src/fuse.rs:64-215; returns points sorted by voxel key."""
    ext = []
    for a in range(3):
        ax = sorted(p[a] for p in sparse)
        n = len(ax)
        ext.append(ax[min(int(n * 0.98), n - 1)] - ax[min(int(n * 0.02), n - 1)])
    diag = np.sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2])
    cell = max(diag * voxel_rel, 1e-9)
    cands = []
    for ri, v in enumerate(views):
        dm = depth_maps[ri]
        if dm is None:
            continue
        R, t = v["R"], v["t"]
        f, cx, cy, k = v["cam"]
        for py in range(v["h"]):
            for px in range(v["w"]):
                zr = float(dm[py, px])
                if zr <= 0.0:
                    continue
                nx, ny = cam_normalize(v["cam"], float(px), float(py))
                xr = [nx * zr, ny * zr, 1.0 * zr]
                xw = _mtv(R, [xr[0] - t[0], xr[1] - t[1], xr[2] - t[2]])
                cons = []
                for si in order[ri]:
                    sv = views[si]
                    xs = _mv(sv["R"], xw)
                    xs = [xs[i] + sv["t"][i] for i in range(3)]
                    if xs[2] <= 1e-6:
                        continue
                    z = xs[2]
                    xn, yn = xs[0] / z, xs[1] / z
                    dd = 1.0 + sv["cam"][3] * (xn * xn + yn * yn)
                    us = sv["cam"][0] * xn * dd + sv["cam"][1]
                    vs = sv["cam"][0] * yn * dd + sv["cam"][2]
                    zs = sample_depth(depth_maps[si], us, vs)
                    if zs <= 0.0:
                        continue
                    if abs((xs[2] - zs) / xs[2]) < depth_diff:
                        a, b = cam_normalize(sv["cam"], us, vs)
                        x2 = [a * zs - sv["t"][0], b * zs - sv["t"][1], 1.0 * zs - sv["t"][2]]
                        cons.append(_mtv(sv["R"], x2))
                if len(cons) < min_consistent:
                    continue
                acc = list(xw)
                for p in cons:
                    acc = [acc[i] + p[i] for i in range(3)]
                m = float(len(cons) + 1)
                acc = [acc[i] / m for i in range(3)]
                g = int(v["gray"][py, px])
                cands.append((acc, (g, g, g)))
    vox = {}
    for p, c in cands:
        key = tuple(int(np.floor(p[a] / cell)) for a in range(3))
        e = vox.setdefault(key, [0.0, 0.0, 0.0, 0, 0, 0, 0])
        for a in range(3):
            e[a] += p[a]
        for a in range(3):
            e[3 + a] = (e[3 + a] + c[a]) & 0xFFFF
        e[6] += 1
    keys = sorted(vox)
    xyz = np.array([[vox[k][a] / vox[k][6] for a in range(3)] for k in keys], np.float64).reshape(-1, 3)
    def round_half_away(x):  # f64::round for x >= 0
        i = int(x)
        return i + (1 if x - i >= 0.5 else 0)

    rgb = np.array([[min(255, round_half_away(vox[k][3 + a] / vox[k][6])) for a in range(3)] for k in keys],
                   np.uint8).reshape(-1, 3)
    return xyz, rgb, len(cands)


def main():
    from rustcolmap_b200 import scene
    sc = scene.corner_room(seed=11, n_views=3, w=40, h=30, f=46.0, arc_deg=24.0, n_patches=40, per_view_sparse=60)
    views = []
    for v in sc.views:
        views.append(dict(w=v.w, h=v.h, cam=(v.cam.f, v.cam.cx, v.cam.cy, v.cam.k),
                          R=[[float(x) for x in row] for row in v.R], t=[float(x) for x in v.t], gray=v.gray))
    census = [census_map(v["gray"]) for v in views]
    zmin, zmax = 2.5, 8.0
    num_hyp, sweeps, cost_thr = 8, 1, 0.38
    out = {}
    depths = []
    for ref, srcs in ((0, [1, 2]), (1, [0, 2]), (2, [1, 0])):
        d, c, n = estimate_depth(views, census, ref, srcs, zmin, zmax, num_hyp, sweeps, cost_thr)
        depths.append(d)
        out[f"depth{ref}"], out[f"cost{ref}"], out[f"normal{ref}"] = d, c, n
        out[f"srcs{ref}"] = np.array(srcs, np.int32)
    # fixed plane field cost KAT on view 0: random slanted planes, mixed hints
    rng = np.random.default_rng(5)
    ws = Workspace(views, census, 0, [1, 2], zmin, zmax)
    h, w = views[0]["h"], views[0]["w"]
    planes = np.zeros((h, w, 4), np.float32)
    hints = np.zeros((h, w), np.float32)
    pcost = np.zeros((h, w), np.float32)
    phs = np.zeros((h, w), np.int32)
    for y in range(h):
        for x in range(w):
            n = rng.normal(size=3) * [0.4, 0.4, 1.0]
            n[2] = abs(n[2]) + 0.2
            n = (n / np.linalg.norm(n)).astype(np.float32)
            dpl = F(rng.uniform(1.5, 9.0))
            hint = F([np.inf, 0.05, 0.2, 0.5][int(rng.integers(0, 4))])
            planes[y, x] = (n[0], n[1], n[2], dpl)
            hints[y, x] = hint
            pcost[y, x], phs[y, x] = plane_cost(ws, x, y, n[0], n[1], n[2], dpl, hint)
    out.update(planes=planes, hints=hints, plane_cost=pcost, plane_hsum=phs)
    # fusion over the three depth maps
    order = [[1, 2], [0, 2], [1, 0]]
    sp = [tuple(p) for p in sc.sparse.xyz.tolist()]
    fx, frgb, ncand = fuse(views, depths, order, sp, 1, 0.03, 0.0015)
    out.update(fused_xyz=fx, fused_rgb=frgb, fused_candidates=np.array(ncand), sparse_xyz=sc.sparse.xyz)
    for i, v in enumerate(views):
        out[f"gray{i}"] = v["gray"]
        out[f"census{i}"] = census[i]
        out[f"cam{i}"] = np.array(v["cam"], np.float64)
        out[f"R{i}"] = np.array(v["R"], np.float64)
        out[f"t{i}"] = np.array(v["t"], np.float64)
    out["zrange"] = np.array([zmin, zmax])
    out["params"] = np.array([num_hyp, sweeps, cost_thr])
    # rng stream KAT
    r = Rng(pixel_rng(3, 5, 9))
    out["rng_seed_3_5_9"] = np.array([pixel_rng(3, 5, 9)], np.uint64)
    out["rng_u64"] = np.array([r.next_u64() for _ in range(4)], np.uint64)
    out["rng_gauss"] = np.array([r.gauss() for _ in range(4)], np.float32)
    np.savez_compressed(os.path.join(HERE, "tiny_corner.npz"), **out)
    print("wrote tiny_corner.npz;", "valid px:", [int((d > 0).sum()) for d in depths], "fused:", len(fx))


if __name__ == "__main__":
    main()
