"""Seeded synthetic scenes with analytic ground truth for the dense-MVS path.

The reference has no synthetic MVS scene (its demo scene is for SfM only), so
these generators are this project's own.  Each returns views at working
resolution, ground-truth depth (z in the camera; 0 = no surface) and a sparse
model whose tracks come from visibility in the ground truth, so run_mvs-style
co-visibility, support-view selection and depth ranges work as they do on a
real COLMAP model.

corner_room  — floor + 3 walls, value noise + flat rectangles, cameras on an arc
orbit_room   — 4-wall room + boxes (+ spheres), cameras on a full orbit;
               per-view image sizes may differ
"""
import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _lib
from .types import Cam, SparseModel, ViewData


class Prim(C.Structure):
    _fields_ = [("kind", C.c_int32), ("tex_seed", C.c_int32), ("tex_freq", C.c_float), ("tex_lo", C.c_float),
                ("tex_hi", C.c_float), ("p", C.c_float * 11)]


class Patch(C.Structure):
    _fields_ = [("prim", C.c_int32), ("u0", C.c_float), ("v0", C.c_float), ("u1", C.c_float), ("v1", C.c_float),
                ("value", C.c_float)]


class RCam(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("f", C.c_double), ("cx", C.c_double), ("cy", C.c_double),
                ("R", C.c_double * 9), ("t", C.c_double * 3)]


RECT, BOX, SPHERE = 0, 1, 2


@dataclass
class SyntheticScene:
    views: List[ViewData]
    gt_depth: List[np.ndarray]
    gt_normal: Optional[List[np.ndarray]]
    sparse: SparseModel
    name: str
    seed: int
    prims: Optional[list] = None  # the analytic surfaces the views were rendered from


def look_at(eye, target, up=(0.0, 0.0, 1.0)):
    """World->camera (R, t) of a camera at `eye` looking at `target`, with
    x right, y down, z forward."""
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    R = np.stack([right, down, fwd])
    return R, -R @ eye


def _rect(o, u, v, U, V, rng, freq=9.0):
    p = Prim()
    p.kind = RECT
    p.tex_seed = int(rng.integers(1, 1 << 30))
    p.tex_freq = freq
    p.tex_lo = float(rng.uniform(15, 70))
    p.tex_hi = float(rng.uniform(180, 245))
    vals = list(o) + list(u) + list(v) + [U, V]
    for i, x in enumerate(vals):
        p.p[i] = float(x)
    return p


def _box(lo, hi, rng, freq=12.0):
    p = Prim()
    p.kind = BOX
    p.tex_seed = int(rng.integers(1, 1 << 30))
    p.tex_freq = freq
    p.tex_lo = float(rng.uniform(10, 90))
    p.tex_hi = float(rng.uniform(160, 250))
    for i, x in enumerate(list(lo) + list(hi)):
        p.p[i] = float(x)
    return p


def _sphere(c, r, rng, freq=12.0):
    p = Prim()
    p.kind = SPHERE
    p.tex_seed = int(rng.integers(1, 1 << 30))
    p.tex_freq = freq
    p.tex_lo = float(rng.uniform(10, 90))
    p.tex_hi = float(rng.uniform(160, 250))
    for i, x in enumerate(list(c) + [r]):
        p.p[i] = float(x)
    return p


def _patches(rects_idx, prims, n, rng):
    out = []
    for _ in range(n):
        pi = int(rng.choice(rects_idx))
        U, V = prims[pi].p[9], prims[pi].p[10]
        su, sv = rng.uniform(0.1, 0.8, size=2)
        u0 = rng.uniform(0, max(U - su, 1e-3))
        v0 = rng.uniform(0, max(V - sv, 1e-3))
        q = Patch()
        q.prim, q.u0, q.v0, q.u1, q.v1 = pi, u0, v0, u0 + su, v0 + sv
        q.value = float(rng.integers(0, 256))
        out.append(q)
    return out


_HOST_RENDERER = None


def use_host_renderer(path):
    """Renders through `path`, a host-only build of the same renderer
    (scene.cu compiled as plain C++), instead of librcscene.so: for CPU-only
    programs that must not load the CUDA libraries.  device must then be -1."""
    global _HOST_RENDERER
    L = C.CDLL(path)
    vp, i32 = C.c_void_p, C.c_int32
    L.rcscene_render.argtypes = [vp, i32, vp, i32, vp, i32, i32, i32, vp, vp, vp]
    L.rcscene_render.restype = C.c_int
    L.rcscene_last_error.argtypes = []
    L.rcscene_last_error.restype = C.c_char_p
    _HOST_RENDERER = L


def render(prims, patches, cams, supersample=2, device=-1, normals=False):
    """Ray-cast every camera: returns (gray list, depth list, normal list|None)."""
    L = _HOST_RENDERER if _HOST_RENDERER is not None else _lib.scene()
    pa = (Prim * len(prims))(*prims)
    qa = (Patch * max(1, len(patches)))(*patches) if patches else None
    ca = (RCam * len(cams))(*cams)
    grays = [np.empty((c.h, c.w), np.uint8) for c in cams]
    depths = [np.empty((c.h, c.w), np.float32) for c in cams]
    nrms = [np.empty((c.h, c.w, 3), np.float32) for c in cams] if normals else None
    gp = (C.c_void_p * len(cams))(*[g.ctypes.data for g in grays])
    dp = (C.c_void_p * len(cams))(*[d.ctypes.data for d in depths])
    np_ = (C.c_void_p * len(cams))(*[n.ctypes.data for n in nrms]) if normals else None
    rc = L.rcscene_render(pa, len(prims), qa, len(patches), ca, len(cams), supersample, device, gp, dp, np_)
    if rc != 0:
        raise RuntimeError("rcscene_render failed: " + L.rcscene_last_error().decode())
    return grays, depths, nrms


def _cam(w, h, f, R, t):
    c = RCam()
    c.w, c.h, c.f, c.cx, c.cy = w, h, f, w * 0.5, h * 0.5
    for i, x in enumerate(R.reshape(9)):
        c.R[i] = float(x)
    for i, x in enumerate(t):
        c.t[i] = float(x)
    return c


def sample_sparse(views, depths, rng, per_view=300, rel_tol=0.01):
    """Sparse model from ground truth: per view, back-project random valid
    pixels; a point's track lists every view that sees it unoccluded."""
    pts = []
    for v, d in zip(views, depths):
        ys, xs = np.nonzero(d > 0)
        if len(xs) == 0:
            continue
        k = rng.choice(len(xs), size=min(per_view, len(xs)), replace=False)
        x, y = xs[k].astype(np.float64), ys[k].astype(np.float64)
        z = d[ys[k], xs[k]].astype(np.float64)
        rays = np.stack([(x - v.cam.cx) / v.cam.f * z, (y - v.cam.cy) / v.cam.f * z, z], axis=1)
        pts.append((rays - v.t) @ v.R)  # R^T (z*ray - t)
    X = np.concatenate(pts) if pts else np.zeros((0, 3))
    tracks = [[] for _ in range(len(X))]
    for vi, (v, d) in enumerate(zip(views, depths)):
        Xc = X @ v.R.T + v.t
        z = Xc[:, 2]
        with np.errstate(divide="ignore", invalid="ignore"):
            u = v.cam.f * Xc[:, 0] / z + v.cam.cx
            w = v.cam.f * Xc[:, 1] / z + v.cam.cy
        ok = (z > 1e-6) & (u >= 0) & (w >= 0) & (u <= v.w - 1) & (w <= v.h - 1)
        idx = np.nonzero(ok)[0]
        ui = np.clip(np.rint(u[idx]).astype(np.int64), 0, v.w - 1)
        wi = np.clip(np.rint(w[idx]).astype(np.int64), 0, v.h - 1)
        gz = d[wi, ui].astype(np.float64)
        vis = idx[(gz > 0) & (np.abs(gz - z[idx]) <= rel_tol * z[idx])]
        for p in vis:
            tracks[p].append(vi)
    off = np.zeros(len(X) + 1, np.uint64)
    for i, t in enumerate(tracks):
        off[i + 1] = off[i] + len(t)
    tv = np.array([x for t in tracks for x in t], np.int32)
    return SparseModel(np.ascontiguousarray(X), off, tv)


def _views(cams, grays, name):
    views = []
    for i, (c, g) in enumerate(zip(cams, grays)):
        R = np.array(c.R[:], np.float64).reshape(3, 3)
        t = np.array(c.t[:], np.float64)
        rgb = np.repeat(g[:, :, None], 3, axis=2)
        views.append(ViewData(f"{name}_{i:03d}.png", i, c.w, c.h, Cam(c.f, c.cx, c.cy, 0.0), R, t, g, rgb))
    return views


def corner_room(seed=0, n_views=8, w=384, h=288, f=440.0, arc_deg=60.0, n_patches=200, device=-1,
                normals=False, per_view_sparse=300):
    """Corner room: floor + 3 walls (planes 3-6 units from the cameras),
    4-octave value noise + `n_patches` flat rectangles; `n_views` cameras on
    an `arc_deg` arc facing the corner."""
    rng = np.random.default_rng(seed)
    S, H = 4.0, 4.0
    prims = [
        _rect((-S, -S, 0), (1, 0, 0), (0, 1, 0), 2 * S, 2 * S, rng),  # floor
        _rect((S, -S, 0), (0, 1, 0), (0, 0, 1), 2 * S, H, rng),  # x = +S
        _rect((-S, S, 0), (1, 0, 0), (0, 0, 1), 2 * S, H, rng),  # y = +S
        _rect((-S, -S, 0), (0, 1, 0), (0, 0, 1), 2 * S, H, rng),  # x = -S
    ]
    patches = _patches([0, 1, 2, 3], prims, n_patches, rng)
    target = np.array([3.0, 3.0, 1.1])
    cams = []
    for i in range(n_views):
        a = np.deg2rad(225.0 - arc_deg / 2 + arc_deg * (i / max(n_views - 1, 1)))
        eye = target + 4.4 * np.array([np.cos(a), np.sin(a), 0.0]) + np.array([0, 0, 0.6 + 0.1 * np.sin(3 * a)])
        R, t = look_at(eye, target)
        cams.append(_cam(w, h, f, R, t))
    grays, depths, nrms = render(prims, patches, cams, device=device, normals=normals)
    views = _views(cams, grays, "corner")
    sparse = sample_sparse(views, depths, rng, per_view=per_view_sparse)
    return SyntheticScene(views, depths, nrms, sparse, "corner_room", seed, prims)


def orbit_room(seed=0, n_views=64, sizes=((960, 720),), f_rel=1.1, n_boxes=20, n_spheres=0, n_patches=200,
               device=-1, normals=False, per_view_sparse=300, size_choice=None, arc_deg=360.0):
    """Room with 4 walls + floor, `n_boxes` textured boxes (0.2-1.0 units) and
    `n_spheres` spheres (radius 0.3-0.8) in the middle; `n_views` cameras on a
    full orbit (or an arc of arc_deg degrees) looking inward.  sizes: candidate (w, h); with size_choice
    'random' each view draws one, else all views use sizes[0].  f = f_rel *
    long side."""
    rng = np.random.default_rng(seed)
    S, H = 6.0, 4.0
    prims = [
        _rect((-S, -S, 0), (1, 0, 0), (0, 1, 0), 2 * S, 2 * S, rng),
        _rect((S, -S, 0), (0, 1, 0), (0, 0, 1), 2 * S, H, rng),
        _rect((-S, S, 0), (1, 0, 0), (0, 0, 1), 2 * S, H, rng),
        _rect((-S, -S, 0), (0, 1, 0), (0, 0, 1), 2 * S, H, rng),
        _rect((-S, -S, 0), (1, 0, 0), (0, 0, 1), 2 * S, H, rng),
    ]
    patches = _patches([0, 1, 2, 3, 4], prims, n_patches, rng)
    for _ in range(n_boxes):
        r = 2.6 * np.sqrt(rng.uniform())
        a = rng.uniform(0, 2 * np.pi)
        c = np.array([r * np.cos(a), r * np.sin(a)])
        sz = rng.uniform(0.2, 1.0, size=3)
        lo = np.array([c[0] - sz[0] / 2, c[1] - sz[1] / 2, 0.0])
        hi = np.array([c[0] + sz[0] / 2, c[1] + sz[1] / 2, sz[2]])
        prims.append(_box(lo, hi, rng))
    for _ in range(n_spheres):
        r = 2.6 * np.sqrt(rng.uniform())
        a = rng.uniform(0, 2 * np.pi)
        rad = rng.uniform(0.3, 0.8)
        prims.append(_sphere((r * np.cos(a), r * np.sin(a), rad + rng.uniform(0, 0.8)), rad, rng))
    target = np.array([0.0, 0.0, 0.4])
    cams = []
    for i in range(n_views):
        a = np.deg2rad(arc_deg) * i / (n_views if arc_deg >= 360.0 else max(n_views - 1, 1))
        eye = np.array([4.3 * np.cos(a), 4.3 * np.sin(a), 1.8 + 0.25 * np.sin(5 * a)])
        R, t = look_at(eye, target)
        if size_choice == "random":
            w, h = sizes[int(rng.integers(0, len(sizes)))]
        else:
            w, h = sizes[0]
        cams.append(_cam(w, h, f_rel * max(w, h), R, t))
    grays, depths, nrms = render(prims, patches, cams, device=device, normals=normals)
    views = _views(cams, grays, "orbit")
    sparse = sample_sparse(views, depths, rng, per_view=per_view_sparse)
    return SyntheticScene(views, depths, nrms, sparse, "orbit_room", seed, prims)


def surface_distance(xyz, prims, chunk=65536):
    """Distance of each point (n, 3) to the nearest surface of the scene's
    primitives (rectangles, axis-aligned boxes, spheres), in scene units:
    the ground-truth error of a fused point cloud."""
    xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
    out = np.full(len(xyz), np.inf)
    for a in range(0, len(xyz), chunk):
        p = xyz[a:a + chunk]
        best = np.full(len(p), np.inf)
        for q in prims:
            v = np.array(q.p[:11], np.float64)
            if q.kind == RECT:
                o, u, w, U, V = v[0:3], v[3:6], v[6:9], v[9], v[10]
                d = p - o
                s = np.clip(d @ u, 0.0, U)
                t = np.clip(d @ w, 0.0, V)
                dist = np.linalg.norm(d - s[:, None] * u - t[:, None] * w, axis=1)
            elif q.kind == BOX:
                lo, hi = v[0:3], v[3:6]
                outside = np.linalg.norm(p - np.clip(p, lo, hi), axis=1)
                inside = np.minimum(p - lo, hi - p).min(axis=1)
                dist = np.where(outside > 0, outside, np.abs(inside))
            else:
                dist = np.abs(np.linalg.norm(p - v[0:3], axis=1) - v[3])
            best = np.minimum(best, dist)
        out[a:a + chunk] = best
    return out


def gt_metrics(depth, gt, tol=0.01):
    """Per-pixel error against ground truth: fraction of valid estimates whose
    inverse depth is within `tol` (relative) of the truth (accuracy), and the
    fraction of all pixels with ground truth that are valid and within it
    (completeness)."""
    has_gt = gt > 0
    valid = (depth > 0) & has_gt
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.abs(1.0 / depth[valid] - 1.0 / gt[valid]) * gt[valid]
    good = int((rel <= tol).sum())
    nv = int(valid.sum())
    return {"valid": nv, "gt_pixels": int(has_gt.sum()), "within": good,
            "accuracy": good / nv if nv else 0.0,
            "completeness": good / max(int(has_gt.sum()), 1)}
