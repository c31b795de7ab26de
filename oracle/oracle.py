"""ctypes front-end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module, as the checker.  The product path (rustcolmap_b200) never
does.  The oracle restates the reference `mvs` crate in C++
(oracle/mvs_oracle.cpp); parity with the reference itself is UNPINNED (no
Rust toolchain, no reference golden vectors) — see oracle/mvs_oracle.h.
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

from rustcolmap_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libmvs_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        vp, i32, u64, f32, f64 = C.c_void_p, C.c_int32, C.c_uint64, C.c_float, C.c_double
        L.orc_census_map.argtypes = [vp, i32, i32, vp]
        L.orc_pixel_rng.argtypes = [i32, i32, u64]
        L.orc_pixel_rng.restype = u64
        L.orc_next_u64.argtypes = [vp]
        L.orc_next_u64.restype = u64
        L.orc_uniform.argtypes = [vp]
        L.orc_uniform.restype = f32
        L.orc_gauss.argtypes = [vp]
        L.orc_gauss.restype = f32
        L.orc_f32_to_i32.argtypes = [f32]
        L.orc_f32_to_i32.restype = i32
        L.orc_cam_normalize.argtypes = [f64, f64, f64, f64, f64, f64, vp]
        L.orc_rays.argtypes = [vp, vp, vp]
        L.orc_rel_pose.argtypes = [vp, vp, vp, vp]
        L.orc_plane_cost_field.argtypes = [vp, i32, i32, vp, i32, vp, vp, vp, vp, i32]
        L.orc_estimate_depth.argtypes = [vp, i32, i32, vp, i32, f64, f64, vp, vp, vp, vp, i32, vp]
        L.orc_estimate_depth_seeded.argtypes = [vp, i32, i32, vp, i32, f64, f64, vp, vp, f32, i32, f32, vp, vp,
                                                vp, i32, vp]
        L.orc_logit_threshold.argtypes = [f32]
        L.orc_logit_threshold.restype = f32
        L.orc_fuse_depth_maps.argtypes = [vp, i32, vp, vp, vp, vp, u64, vp, vp, vp, vp, vp, i32]
        L.orc_free.argtypes = [vp]
        L.orc_write_ply_binary.argtypes = [C.c_char_p, vp, vp, u64]
        L.orc_plan.argtypes = [vp, vp, i32, vp, vp, vp, vp, vp, vp]
        L.orc_depth_vis.argtypes = [vp, i32, i32, vp, vp]
        L.orc_depth_vis.restype = None
        L.orc_fuse_candidates.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32]
        L.orc_fuse_reduce.argtypes = [vp, vp, u64, vp, u64, vp, vp, vp, vp]
        L.orc_resize_view.argtypes = [vp, i32, i32, i32, i32, i32, vp, vp]
        L.orc_extract_sift.argtypes = [vp, vp, i32, i32, C.c_uint32, f64, vp, vp, vp, vp, vp]
        L.orc_match_pair.argtypes = [vp, C.c_uint32, vp, C.c_uint32, f64, vp, vp, vp]
        L.orc_match_pair.restype = None
        L.orc_resize_view.restype = None
        _lib = L
    return _lib


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with status {rc}")


def census_map(gray):
    gray = np.ascontiguousarray(gray, dtype=np.uint8)
    h, w = gray.shape
    out = np.empty((h, w), np.uint64)
    lib().orc_census_map(gray.ctypes.data, w, h, out.ctypes.data)
    return out


def pixel_rng(x, y, salt):
    return int(lib().orc_pixel_rng(x, y, salt))


def rng_stream(x, y, salt, n, kind="gauss"):
    s = C.c_uint64(pixel_rng(x, y, salt))
    fn = {"gauss": lib().orc_gauss, "uniform": lib().orc_uniform, "u64": lib().orc_next_u64}[kind]
    return [fn(C.byref(s)) for _ in range(n)]


def f32_to_i32(v):
    return int(lib().orc_f32_to_i32(float(v)))


def cam_normalize(cam, u, v):
    out = np.empty(2, np.float64)
    lib().orc_cam_normalize(*[float(c) for c in cam], float(u), float(v), out.ctypes.data)
    return out


def rays(view):
    va = _abi.view_array([view])
    rx = np.empty((view.h, view.w), np.float32)
    ry = np.empty((view.h, view.w), np.float32)
    lib().orc_rays(C.addressof(va[0]), rx.ctypes.data, ry.ctypes.data)
    return rx, ry


def rel_pose(ref, src):
    va = _abi.view_array([ref, src])
    rs = np.empty(9, np.float32)
    ts = np.empty(3, np.float32)
    lib().orc_rel_pose(C.addressof(va[0]), C.addressof(va[1]), rs.ctypes.data, ts.ctypes.data)
    return rs, ts


def plane_cost_field(views, ref_idx, srcs, planes, hints, nthreads=0):
    va = _abi.view_array(views)
    srcs = np.ascontiguousarray(srcs, dtype=np.int32)
    r = views[ref_idx]
    planes = np.ascontiguousarray(planes, dtype=np.float32).reshape(r.h, r.w, 4)
    hints = np.ascontiguousarray(hints, dtype=np.float32).reshape(r.h, r.w)
    cost = np.empty((r.h, r.w), np.float32)
    hsum = np.empty((r.h, r.w), np.int32)
    rc = lib().orc_plane_cost_field(va, len(views), ref_idx, srcs.ctypes.data, len(srcs),
                                    planes.ctypes.data, hints.ctypes.data, cost.ctypes.data,
                                    hsum.ctypes.data, nthreads)
    _chk(rc, "plane_cost_field")
    return cost, hsum


def estimate_depth(views, ref_idx, srcs, zmin, zmax, opts, nthreads=0, normals=True):
    """stereo::estimate_depth on the CPU.  Returns (depth, cost, normal|None, work)."""
    va = _abi.view_array(views)
    srcs = np.ascontiguousarray(srcs, dtype=np.int32)
    r = views[ref_idx]
    depth = np.empty((r.h, r.w), np.float32)
    cost = np.empty((r.h, r.w), np.float32)
    normal = np.empty((r.h, r.w, 3), np.float32) if normals else None
    work = np.zeros(2, np.uint64)
    o = opts.to_c()
    rc = lib().orc_estimate_depth(va, len(views), ref_idx, srcs.ctypes.data, len(srcs), float(zmin),
                                  float(zmax), C.byref(o), depth.ctypes.data, cost.ctypes.data,
                                  _abi.ptr(normal), nthreads, work.ctypes.data)
    _chk(rc, "estimate_depth")
    return depth, cost, normal, (int(work[0]), int(work[1]))


def estimate_depth_seeded(views, ref_idx, srcs, zmin, zmax, opts, pred, conf_thr, n_local=1, span=0.0,
                          nthreads=0, normals=True):
    """estimate_depth with the learned init (no reference counterpart): pred
    is the reference view's (h/4, w/4, 16) f32 prediction map.  Returns
    (depth, cost, normal|None, seeded pixel count)."""
    va = _abi.view_array(views)
    srcs = np.ascontiguousarray(srcs, dtype=np.int32)
    r = views[ref_idx]
    pred = np.ascontiguousarray(pred, dtype=np.float32)
    assert pred.size == (r.h // 4) * (r.w // 4) * 16
    if pred.size == 0:
        pred = np.zeros(16, np.float32)
    depth = np.empty((r.h, r.w), np.float32)
    cost = np.empty((r.h, r.w), np.float32)
    normal = np.empty((r.h, r.w, 3), np.float32) if normals else None
    seeded = C.c_uint64()
    o = opts.to_c()
    rc = lib().orc_estimate_depth_seeded(va, len(views), ref_idx, srcs.ctypes.data, len(srcs), float(zmin),
                                         float(zmax), C.byref(o), pred.ctypes.data, float(conf_thr), int(n_local),
                                         float(span), depth.ctypes.data, cost.ctypes.data, _abi.ptr(normal),
                                         nthreads, C.byref(seeded))
    _chk(rc, "estimate_depth_seeded")
    return depth, cost, normal, seeded.value


def logit_threshold(conf_thr):
    return float(lib().orc_logit_threshold(float(conf_thr)))


def fuse_depth_maps(views, depth_maps, order_offsets, order, sparse_xyz, opts, nthreads=0):
    """fuse::fuse_depth_maps on the CPU.  depth_maps: list of (h, w) f32 or
    None.  Returns (xyz (n,3) f64, rgb (n,3) u8, n_candidates), sorted by
    voxel key."""
    va = _abi.view_array(views)
    dms = [None if d is None else np.ascontiguousarray(d, dtype=np.float32) for d in depth_maps]
    dptr = (C.c_void_p * len(views))(*[None if d is None else d.ctypes.data for d in dms])
    off = np.ascontiguousarray(order_offsets, dtype=np.int32)
    ordr = np.ascontiguousarray(order, dtype=np.int32)
    if ordr.size == 0:
        ordr = np.zeros(1, np.int32)
    sp = np.ascontiguousarray(sparse_xyz, dtype=np.float64)
    xyz_p, rgb_p = C.c_void_p(), C.c_void_p()
    n = C.c_uint64()
    ncand = C.c_uint64()
    o = opts.to_c()
    rc = lib().orc_fuse_depth_maps(va, len(views), dptr, off.ctypes.data, ordr.ctypes.data,
                                   sp.ctypes.data, len(sp), C.byref(o), C.byref(xyz_p),
                                   C.byref(rgb_p), C.byref(n), C.byref(ncand), nthreads)
    _chk(rc, "fuse_depth_maps")
    nn = n.value
    xyz = np.ctypeslib.as_array((C.c_double * (3 * max(nn, 1))).from_address(xyz_p.value))[: 3 * nn]
    rgb = np.ctypeslib.as_array((C.c_uint8 * (3 * max(nn, 1))).from_address(rgb_p.value))[: 3 * nn]
    xyz = xyz.reshape(nn, 3).copy()
    rgb = rgb.reshape(nn, 3).copy()
    lib().orc_free(xyz_p)
    lib().orc_free(rgb_p)
    return xyz, rgb, ncand.value


def depth_vis(depth):
    """fuse::save_depth_vis's image on the CPU: ((h, w) u8, lo, hi)."""
    d = np.ascontiguousarray(depth, dtype=np.float32)
    h, w = d.shape
    out = np.empty((h, w), np.uint8)
    lh = np.zeros(2, np.float32)
    lib().orc_depth_vis(d.ctypes.data, w, h, out.ctypes.data, lh.ctypes.data)
    return out, float(lh[0]), float(lh[1])


def resize_view(img, mw, mh):
    """load_views' image preparation on the CPU (lib.rs:183-194): (h, w) or
    (h, w, c) u8 -> ((mh, mw) grey, (mh, mw, 3) RGB)."""
    a = np.ascontiguousarray(img, dtype=np.uint8)
    if a.ndim == 2:
        a = a[:, :, None]
    h, w, c = a.shape
    gray = np.empty((mh, mw), np.uint8)
    rgb = np.empty((mh, mw, 3), np.uint8)
    lib().orc_resize_view(a.ctypes.data, w, h, c, mw, mh, gray.ctypes.data, rgb.ctypes.data)
    return gray, rgb


def _take(xyz_p, rgb_p, nn):
    xyz = np.ctypeslib.as_array((C.c_double * (3 * max(nn, 1))).from_address(xyz_p.value))[: 3 * nn]
    rgb = np.ctypeslib.as_array((C.c_uint8 * (3 * max(nn, 1))).from_address(rgb_p.value))[: 3 * nn]
    xyz = xyz.reshape(nn, 3).copy()
    rgb = rgb.reshape(nn, 3).copy()
    lib().orc_free(xyz_p)
    lib().orc_free(rgb_p)
    return xyz, rgb


def fuse_candidates(views, depth_maps, order_offsets, order, ref_views, opts, nthreads=0):
    """The consistency half of fuse_depth_maps for the pixels of ref_views:
    (xyz (n,3) f64, rgb (n,3) u8, per-view counts), view-then-pixel order."""
    va = _abi.view_array(views)
    dms = [None if d is None else np.ascontiguousarray(d, dtype=np.float32) for d in depth_maps]
    dptr = (C.c_void_p * len(views))(*[None if d is None else d.ctypes.data for d in dms])
    off = np.ascontiguousarray(order_offsets, dtype=np.int32)
    ordr = np.ascontiguousarray(order, dtype=np.int32)
    if ordr.size == 0:
        ordr = np.zeros(1, np.int32)
    mask = np.zeros(len(views), np.uint8)
    mask[list(ref_views)] = 1
    per_view = np.zeros(len(views), np.uint64)
    xyz_p, rgb_p = C.c_void_p(), C.c_void_p()
    n = C.c_uint64()
    o = opts.to_c()
    rc = lib().orc_fuse_candidates(va, len(views), dptr, off.ctypes.data, ordr.ctypes.data, mask.ctypes.data,
                                   C.byref(o), C.byref(xyz_p), C.byref(rgb_p), C.byref(n), per_view.ctypes.data,
                                   nthreads)
    _chk(rc, "fuse_candidates")
    xyz, rgb = _take(xyz_p, rgb_p, n.value)
    return xyz, rgb, per_view


def fuse_reduce(xyz, rgb, sparse_xyz, opts):
    """The voxel-dedup half of fuse_depth_maps over candidates in order."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1, 3)
    sp = np.ascontiguousarray(sparse_xyz, dtype=np.float64)
    xyz_p, rgb_p = C.c_void_p(), C.c_void_p()
    n = C.c_uint64()
    o = opts.to_c()
    rc = lib().orc_fuse_reduce(xyz.ctypes.data, rgb.ctypes.data, len(xyz), sp.ctypes.data, len(sp), C.byref(o),
                               C.byref(xyz_p), C.byref(rgb_p), C.byref(n))
    _chk(rc, "fuse_reduce")
    return _take(xyz_p, rgb_p, n.value)


def extract_sift(gray, rgb, max_features=2048, contrast_thr=0.0067):
    """extract_sift on an image at working resolution: (pts (n,2) f64,
    desc (n,128) f32, colors (n,3) u8, n_raw)."""
    g = np.ascontiguousarray(gray, dtype=np.uint8)
    c = np.ascontiguousarray(rgb, dtype=np.uint8)
    h, w = g.shape
    pp, dp, cp = C.c_void_p(), C.c_void_p(), C.c_void_p()
    n, nraw = C.c_uint64(), C.c_uint64()
    _chk(lib().orc_extract_sift(g.ctypes.data, c.ctypes.data, w, h, max_features, contrast_thr, C.byref(pp),
                                C.byref(dp), C.byref(cp), C.byref(n), C.byref(nraw)), "extract_sift")
    k = n.value
    pts = np.ctypeslib.as_array((C.c_double * (2 * max(k, 1))).from_address(pp.value))[: 2 * k].reshape(k, 2).copy()
    desc = np.ctypeslib.as_array((C.c_float * (128 * max(k, 1))).from_address(dp.value))[: 128 * k]
    desc = desc.reshape(k, 128).copy()
    col = np.ctypeslib.as_array((C.c_uint8 * (3 * max(k, 1))).from_address(cp.value))[: 3 * k].reshape(k, 3).copy()
    for p in (pp, dp, cp):
        lib().orc_free(p)
    return pts, desc, col, nraw.value


def match_pair(da, db, ratio=0.8):
    """match_pair of two descriptor sets: (a indices, b indices) u32."""
    a = np.ascontiguousarray(da, dtype=np.float32).reshape(-1, 128)
    b = np.ascontiguousarray(db, dtype=np.float32).reshape(-1, 128)
    k = max(min(len(a), len(b)), 1)
    oa, ob = np.zeros(k, np.uint32), np.zeros(k, np.uint32)
    n = C.c_uint64()
    lib().orc_match_pair(a.ctypes.data, len(a), b.ctypes.data, len(b), ratio, oa.ctypes.data, ob.ctypes.data,
                         C.byref(n))
    return oa[: n.value].copy(), ob[: n.value].copy()


def write_ply_binary(path, xyz, rgb):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    _chk(lib().orc_write_ply_binary(path.encode(), xyz.ctypes.data, rgb.ctypes.data, len(xyz)),
         "write_ply_binary")


def plan(sparse, views, opts):
    """Host glue of run_mvs: returns (sources list, zrange (n,2), fusion order list)."""
    n = len(views)
    va = _abi.view_array(views)
    sp = sparse.to_c()
    so = np.zeros(n + 1, np.int32)
    ss = np.zeros(max(1, n * opts.num_sources), np.int32)
    zr = np.zeros((n, 2), np.float64)
    fo = np.zeros(n + 1, np.int32)
    ff = np.zeros(max(1, n * n), np.int32)
    o = opts.to_c()
    rc = lib().orc_plan(C.byref(sp), va, n, C.byref(o), so.ctypes.data, ss.ctypes.data,
                        zr.ctypes.data, fo.ctypes.data, ff.ctypes.data)
    _chk(rc, "plan")
    srcs = [ss[so[i]:so[i + 1]].tolist() for i in range(n)]
    fus = [ff[fo[i]:fo[i + 1]].tolist() for i in range(n)]
    return srcs, zr, fus


def web_json(xyz, rgb, cap=400_000):
    """dense_web.json of run_mvs (mvs/src/lib.rs:434-485) in plain Python
    floats (IEEE f64): the centroid as sequential sums, the robust radius
    from the sorted distances, stride decimation of the kept points in the
    cloud's order, 4-decimal positions.  None for an empty cloud."""
    pts = [tuple(float(c) for c in p) for p in xyz]
    n = len(pts)
    if n == 0:
        return None
    cx = cy = cz = 0.0
    for p in pts:
        cx += p[0]
    for p in pts:
        cy += p[1]
    for p in pts:
        cz += p[2]
    cx, cy, cz = cx / n, cy / n, cz / n
    dist = [math.sqrt((p[0] - cx) * (p[0] - cx) + (p[1] - cy) * (p[1] - cy) + (p[2] - cz) * (p[2] - cz))
            for p in pts]
    sd = sorted(dist)
    med = sd[n // 2]
    p95 = sd[min(int(n * 0.95), n - 1)]
    r_keep = med + 6.0 * max(abs(p95 - med), max(med, 1e-9) * 0.5)
    kept = [i for i in range(n) if dist[i] <= r_keep]
    stride = -(-len(kept) // cap)
    web = kept[::stride]
    pos = ",".join("[%.4f,%.4f,%.4f]" % pts[i] for i in web)
    col = ",".join("[%d, %d,%d]" % tuple(int(c) for c in rgb[i]) for i in web)
    return '{"n":' + str(len(web)) + ',"pos":[' + pos + '],"col":[' + col + ']}'
