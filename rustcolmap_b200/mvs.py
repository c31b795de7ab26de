"""Host-side mirror of the reference `mvs` crate's public API, running on the
B200 kernels of librcmvs through its C ABI (include/rcmvs.h).

Reference                                   here
mvs::run_mvs            (lib.rs:294)        run_mvs
stereo::estimate_depth  (stereo.rs:234)     estimate_depth / estimate_depth_batch
fuse::fuse_depth_maps   (fuse.rs:64)        fuse_depth_maps
fuse::write_ply_binary  (fuse.rs:222)       write_ply_binary
census_map              (lib.rs:119)        census_map
covisibility/sources/depth_range_for/fusion order (lib.rs:224-418)   plan

Argument meaning and error behaviour follow the reference: estimate_depth
and fuse_depth_maps cannot fail on valid input; run_mvs raises where the
reference returns Err (fewer than 2 views, fewer than 8 sparse points).
There is no CPU path: a missing library or a CUDA error raises RcmvsError.
"""
import ctypes as C
import os
import time

import numpy as np

from . import _abi, _lib
from ._lib import RcmvsError
from .types import DepthMap, MvsOptions, MvsStats, SparseModel, ViewData  # noqa: F401


class Context:
    """One rcmvs_ctx: a CUDA device + stream.  Not thread-safe."""

    def __init__(self, device=0):
        self._L = _lib.mvs()
        p = C.c_void_p()
        rc = self._L.rcmvs_ctx_create(int(device), C.byref(p))
        if rc != 0:
            raise RcmvsError(rc, f"cannot create a context on CUDA device {device} "
                                 "(needs an sm_100 GPU)")
        self.ptr = p
        self.device = device

    def check(self, rc):
        if rc != 0:
            raise RcmvsError(rc, self._L.rcmvs_last_error(self.ptr).decode())

    @property
    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return self._L.rcmvs_ctx_stream(self.ptr)

    def synchronize(self):
        self.check(self._L.rcmvs_ctx_synchronize(self.ptr))

    def diag_wait_timeout(self, limit_ns):
        """Queues the bounded-wait diagnostic (rcmvs_diag_wait_timeout): the
        next synchronize() raises, reporting the timed-out wait."""
        self.check(self._L.rcmvs_diag_wait_timeout(self.ptr, int(limit_ns)))

    def last_work(self):
        e, r = C.c_uint64(), C.c_uint64()
        self.check(self._L.rcmvs_last_work(self.ptr, C.byref(e), C.byref(r)))
        return e.value, r.value

    def timing(self, enable=True):
        """Start (or stop) recording CUDA-event spans around each kernel launch."""
        self.check(self._L.rcmvs_ctx_timing(self.ptr, int(bool(enable))))

    def kernel_time(self, name):
        """(total ms, launches) of kernel `name` since timing was enabled."""
        ms, n = C.c_double(), C.c_uint64()
        self.check(self._L.rcmvs_ctx_kernel_time(self.ptr, name.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def tune_table(self):
        """Tile shapes the autotuner chose on this context, per resolution class."""
        buf = (_abi.TuneEntry * 64)()
        n = C.c_int32()
        self.check(self._L.rcmvs_tune_table(self.ptr, buf, 64, C.byref(n)))
        return [dict(w=e.w, h=e.h, tile_w=e.tile_w, tile_h=e.tile_h, threads_per_pixel=e.threads_per_pixel,
                     ms_best=e.ms_best, ms_default=e.ms_default) for e in buf[:n.value]]

    def set_tune_table(self, entries):
        """Loads a tile-shape table (dicts as returned by tune_table)."""
        buf = (_abi.TuneEntry * max(len(entries), 1))()
        for i, e in enumerate(entries):
            buf[i] = _abi.TuneEntry(e["w"], e["h"], e["tile_w"], e["tile_h"], e.get("threads_per_pixel", 1), 0,
                                    e.get("ms_best", 0.0), e.get("ms_default", 0.0))
        self.check(self._L.rcmvs_tune_set(self.ptr, buf, len(entries)))

    def close(self):
        if getattr(self, "ptr", None):
            self._L.rcmvs_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = {}


def default_context(device=0):
    if device not in _default:
        _default[device] = Context(device)
    return _default[device]


def _ctx(ctx):
    return ctx if ctx is not None else default_context()


def census_map(gray, ctx=None):
    """7x7 census (lib.rs:119-142) of a (h, w) u8 image -> (h, w) u64."""
    ctx = _ctx(ctx)
    gray = np.ascontiguousarray(gray, dtype=np.uint8)
    h, w = gray.shape
    out = np.empty((h, w), np.uint64)
    ctx.check(ctx._L.rcmvs_census(ctx.ptr, gray.ctypes.data, w, h, out.ctypes.data))
    return out


def estimate_depth(views, ref_idx, srcs, zmin, zmax, opts, ctx=None, normals=False):
    """stereo::estimate_depth (stereo.rs:234-394) on the GPU."""
    return estimate_depth_batch(views, [(ref_idx, srcs, zmin, zmax)], opts, ctx, normals)[0]


def estimate_depth_batch(views, jobs, opts, ctx=None, normals=False):
    """Many estimate_depth calls in one batched launch sequence.
    jobs: list of (ref_idx, srcs, zmin, zmax)."""
    ctx = _ctx(ctx)
    va = _abi.view_array(views)
    cj = (_abi.Job * len(jobs))()
    outs = (_abi.DepthOut * len(jobs))()
    keep, res = [], []
    for i, (ref, srcs, zmin, zmax) in enumerate(jobs):
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        r = views[ref]
        d = np.empty((r.h, r.w), np.float32)
        c = np.empty((r.h, r.w), np.float32)
        n = np.empty((r.h, r.w, 3), np.float32) if normals else None
        keep += [s]
        cj[i] = _abi.Job(int(ref), len(s), s.ctypes.data if len(s) else None, float(zmin), float(zmax))
        outs[i] = _abi.DepthOut(d.ctypes.data, c.ctypes.data, _abi.ptr(n))
        res.append(DepthMap(d, c, n))
    o = opts.to_c()
    ctx.check(ctx._L.rcmvs_estimate_depth_batch(ctx.ptr, va, len(views), cj, len(jobs), C.byref(o), outs))
    return res


def _csr(lists):
    off = np.zeros(len(lists) + 1, np.int32)
    for i, l in enumerate(lists):
        off[i + 1] = off[i] + len(l)
    flat = np.array([x for l in lists for x in l] or [0], np.int32)
    return off, flat


def fuse_depth_maps(views, depth_maps, sources, sparse_xyz, opts, ctx=None):
    """fuse::fuse_depth_maps (fuse.rs:64-215) on the GPU.  depth_maps: list of
    DepthMap / (h, w) f32 / None; sources: per-view fusion order lists.
    Returns (xyz (n, 3) f64, rgb (n, 3) u8) sorted by voxel key."""
    ctx = _ctx(ctx)
    va = _abi.view_array(views)
    dms = []
    for d in depth_maps:
        if d is None:
            dms.append(None)
        else:
            dms.append(np.ascontiguousarray(d.depth if isinstance(d, DepthMap) else d, dtype=np.float32))
    dptr = (C.c_void_p * len(views))(*[None if d is None else d.ctypes.data for d in dms])
    off, flat = _csr(sources)
    sp = np.ascontiguousarray(sparse_xyz, dtype=np.float64).reshape(-1, 3)
    pts = _abi.Points()
    o = opts.to_c()
    ctx.check(ctx._L.rcmvs_fuse_depth_maps(ctx.ptr, va, len(views), dptr, off.ctypes.data, flat.ctypes.data,
                                           sp.ctypes.data, len(sp), C.byref(o), C.byref(pts)))
    return _take_points(ctx, pts)


def _take_points(ctx, pts):
    n = pts.n
    if n == 0:
        ctx._L.rcmvs_points_free(C.byref(pts))
        return np.zeros((0, 3), np.float64), np.zeros((0, 3), np.uint8)
    xyz = np.ctypeslib.as_array((C.c_double * (3 * n)).from_address(pts.xyz)).reshape(n, 3).copy()
    rgb = np.ctypeslib.as_array((C.c_uint8 * (3 * n)).from_address(pts.rgb)).reshape(n, 3).copy()
    ctx._L.rcmvs_points_free(C.byref(pts))
    return xyz, rgb


def fuse_candidates(views, depth_maps, sources, ref_views, opts, ctx=None):
    """The consistency half of fuse_depth_maps (fuse.rs:96-167) for the
    pixels of ref_views only.  Returns (xyz (n, 3) f64, rgb (n, 3) u8,
    per-view counts (n_views,) u64), candidates in view-then-pixel order."""
    ctx = _ctx(ctx)
    va = _abi.view_array(views)
    dms = [None if d is None else np.ascontiguousarray(d.depth if isinstance(d, DepthMap) else d, dtype=np.float32)
           for d in depth_maps]
    dptr = (C.c_void_p * len(views))(*[None if d is None else d.ctypes.data for d in dms])
    off, flat = _csr(sources)
    refs = np.array(list(ref_views) or [0], np.int32)
    per_view = np.zeros(len(views), np.uint64)
    pts = _abi.Points()
    o = opts.to_c()
    ctx.check(ctx._L.rcmvs_fuse_candidates(ctx.ptr, va, len(views), dptr, off.ctypes.data, flat.ctypes.data,
                                           refs.ctypes.data, len(ref_views), C.byref(o), C.byref(pts),
                                           per_view.ctypes.data))
    xyz, rgb = _take_points(ctx, pts)
    return xyz, rgb, per_view


def fuse_reduce(xyz, rgb, sparse_xyz, opts, ctx=None):
    """The voxel-dedup half of fuse_depth_maps (fuse.rs:72-92, 176-214) over
    candidates in the reference's accumulation order.  Returns (xyz, rgb)
    sorted by voxel key."""
    ctx = _ctx(ctx)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1, 3)
    sp = np.ascontiguousarray(sparse_xyz, dtype=np.float64).reshape(-1, 3)
    pts = _abi.Points()
    o = opts.to_c()
    ctx.check(ctx._L.rcmvs_fuse_reduce(ctx.ptr, xyz.ctypes.data, rgb.ctypes.data, len(xyz), sp.ctypes.data, len(sp),
                                       C.byref(o), C.byref(pts)))
    return _take_points(ctx, pts)


def depth_vis(depth, ctx=None):
    """fuse::save_depth_vis's image (fuse.rs:241-268) on the GPU: returns
    ((h, w) u8, lo, hi)."""
    ctx = _ctx(ctx)
    d = np.ascontiguousarray(depth, dtype=np.float32)
    h, w = d.shape
    out = np.empty((h, w), np.uint8)
    lh = np.zeros(2, np.float32)
    ctx.check(ctx._L.rcmvs_depth_vis(ctx.ptr, d.ctypes.data, w, h, out.ctypes.data, lh.ctypes.data))
    return out, float(lh[0]), float(lh[1])


def working_size(w, h, max_dim):
    """Working resolution of a w x h camera (lib.rs:155-157, :185-187)."""
    mw, mh = C.c_int32(), C.c_int32()
    rc = _lib.mvs().rcmvs_working_size(w, h, max_dim, C.byref(mw), C.byref(mh))
    if rc != 0:
        raise RcmvsError(rc, f"working_size: bad size {w}x{h}")
    return mw.value, mh.value


def resize_view(img, mw, mh, ctx=None):
    """load_views' image preparation (lib.rs:183-194) on the GPU: the `image`
    crate's Triangle resize_exact to (mw, mh) when the size differs, then
    to_luma8 / to_rgb8.  (h, w) or (h, w, c) u8 -> ((mh, mw) grey,
    (mh, mw, 3) RGB)."""
    ctx = _ctx(ctx)
    a = np.ascontiguousarray(img, dtype=np.uint8)
    if a.ndim == 2:
        a = a[:, :, None]
    h, w, c = a.shape
    if mw <= 0 or mh <= 0:
        raise RcmvsError(-1, f"resize_view: bad size {mw}x{mh}")
    gray = np.empty((mh, mw), np.uint8)
    rgb = np.empty((mh, mw, 3), np.uint8)
    ctx.check(ctx._L.rcmvs_resize_view(ctx.ptr, a.ctypes.data, w, h, c, mw, mh, gray.ctypes.data,
                                       rgb.ctypes.data))
    return gray, rgb


def write_png_gray(path, img):
    """8-bit greyscale PNG (the file save_depth_vis writes)."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape
    rc = _lib.mvs().rcmvs_write_png_gray(os.fsencode(path), img.ctypes.data, w, h)
    if rc != 0:
        raise RcmvsError(rc, f"cannot write {path}")


def _vis_stem(name):
    """Path::file_stem of the view's image name, or "view" (fuse.rs:260-263)."""
    stem = os.path.splitext(os.path.basename(name or ""))[0] if name else ""
    return stem or "view"


def write_ply_binary(path, xyz, rgb):
    """fuse::write_ply_binary (fuse.rs:222-239)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    rc = _lib.mvs().rcmvs_write_ply_binary(os.fsencode(path), xyz.ctypes.data, rgb.ctypes.data, len(xyz))
    if rc != 0:
        raise RcmvsError(rc, f"cannot write {path}")


def plan(sparse, views, opts):
    """Host glue of run_mvs: (sources per view, zrange (n, 2), fusion order per view)."""
    n = len(views)
    va = _abi.view_array(views)
    sp = sparse.to_c()
    so = np.zeros(n + 1, np.int32)
    ss = np.zeros(max(1, n * opts.num_sources), np.int32)
    zr = np.zeros((n, 2), np.float64)
    fo = np.zeros(n + 1, np.int32)
    ff = np.zeros(max(1, n * n), np.int32)
    o = opts.to_c()
    rc = _lib.mvs().rcmvs_plan(C.byref(sp), va, n, C.byref(o), so.ctypes.data, ss.ctypes.data, zr.ctypes.data,
                               fo.ctypes.data, ff.ctypes.data)
    if rc != 0:
        raise RcmvsError(rc, "plan failed (need >= 8 sparse points)")
    return ([ss[so[i]:so[i + 1]].tolist() for i in range(n)], zr,
            [ff[fo[i]:fo[i + 1]].tolist() for i in range(n)])


def plane_cost_field(views, ref_idx, srcs, planes, hints, ctx=None):
    """plane_cost (stereo.rs:158-228) at every pixel for a given plane field
    (h, w, 4) = (nx, ny, nz, d) and hints (h, w).  Returns (cost, hsum)."""
    ctx = _ctx(ctx)
    va = _abi.view_array(views)
    s = np.ascontiguousarray(srcs, dtype=np.int32)
    r = views[ref_idx]
    planes = np.ascontiguousarray(planes, dtype=np.float32).reshape(r.h, r.w, 4)
    hints = np.ascontiguousarray(hints, dtype=np.float32).reshape(r.h, r.w)
    cost = np.empty((r.h, r.w), np.float32)
    hsum = np.empty((r.h, r.w), np.int32)
    ctx.check(ctx._L.rcmvs_plane_cost_field(ctx.ptr, va, len(views), ref_idx, s.ctypes.data if len(s) else None,
                                            len(s), planes.ctypes.data, hints.ctypes.data, cost.ctypes.data,
                                            hsum.ctypes.data))
    return cost, hsum


def selftest_f2i(values, ctx=None):
    ctx = _ctx(ctx)
    v = np.ascontiguousarray(values, dtype=np.float32)
    out = np.empty(len(v), np.int32)
    ctx.check(ctx._L.rcmvs_selftest_f2i(ctx.ptr, v.ctypes.data, len(v), out.ctypes.data))
    return out


def _jobs_c(jobs):
    """(ref, srcs, zmin, zmax) tuples -> rcmvs_job array (+ the arrays it points into)."""
    cj = (_abi.Job * max(len(jobs), 1))()
    keep = []
    for i, (ref, srcs, zmin, zmax) in enumerate(jobs):
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        keep.append(s)
        cj[i] = _abi.Job(int(ref), len(s), s.ctypes.data if len(s) else None, float(zmin), float(zmax))
    return cj, keep


class DeviceScene:
    """Views resident in device memory (rcmvs_scene): census, rays, planes,
    depth maps and the fused cloud never leave HBM between calls."""

    def __init__(self, views, ctx=None):
        self.ctx = _ctx(ctx)
        self.views = views
        self._va = _abi.view_array(views)
        p = C.c_void_p()
        self.ctx.check(self.ctx._L.rcmvs_scene_create(self.ctx.ptr, self._va, len(views), C.byref(p)))
        self.ptr = p
        self.n_points = 0

    def prepare(self):
        self.ctx.check(self.ctx._L.rcmvs_scene_prepare(self.ctx.ptr, self.ptr))

    def estimate(self, jobs, opts):
        cj, keep = _jobs_c(jobs)
        o = opts.to_c()
        self.ctx.check(self.ctx._L.rcmvs_scene_estimate_depth(self.ctx.ptr, self.ptr, cj, len(jobs), C.byref(o)))

    def autotune(self, jobs, opts):
        """Tunes the tile shape of every resolution class of `jobs` not yet
        tuned on this context (rcmvs_autotune); returns the context's table
        as a list of dicts."""
        cj, keep = _jobs_c(jobs)
        o = opts.to_c()
        self.ctx.check(self.ctx._L.rcmvs_autotune(self.ctx.ptr, self.ptr, cj, len(jobs), C.byref(o)))
        return self.ctx.tune_table()

    def depth_vis(self, v):
        """save_depth_vis's image of view v's device-resident depth map:
        ((h, w) u8, lo, hi)."""
        vw = self.views[v]
        out = np.empty((vw.h, vw.w), np.uint8)
        lh = np.zeros(2, np.float32)
        self.ctx.check(self.ctx._L.rcmvs_scene_depth_vis(self.ctx.ptr, self.ptr, int(v), out.ctypes.data,
                                                         lh.ctypes.data))
        return out, float(lh[0]), float(lh[1])

    def fuse(self, fusion_order, sparse_xyz, opts):
        off, flat = _csr(fusion_order)
        sp = np.ascontiguousarray(sparse_xyz, dtype=np.float64).reshape(-1, 3)
        n = C.c_uint64()
        o = opts.to_c()
        self.ctx.check(self.ctx._L.rcmvs_scene_fuse(self.ctx.ptr, self.ptr, off.ctypes.data, flat.ctypes.data,
                                                    sp.ctypes.data, len(sp), C.byref(o), C.byref(n)))
        self.n_points = n.value
        return self.n_points

    def fuse_candidates(self, fusion_order, ref_views, opts):
        """fuse_candidates on the scene's device-resident depth maps."""
        off, flat = _csr(fusion_order)
        refs = np.array(list(ref_views) or [0], np.int32)
        per_view = np.zeros(len(self.views), np.uint64)
        pts = _abi.Points()
        o = opts.to_c()
        self.ctx.check(self.ctx._L.rcmvs_scene_fuse_candidates(self.ctx.ptr, self.ptr, off.ctypes.data,
                                                               flat.ctypes.data, refs.ctypes.data, len(ref_views),
                                                               C.byref(o), C.byref(pts), per_view.ctypes.data))
        xyz, rgb = _take_points(self.ctx, pts)
        return xyz, rgb, per_view

    # device-to-device moves (one scene over several processes); ptr
    # arguments are device addresses (e.g. torch CUDA tensors' data_ptr())
    def depth_to_device(self, v, ptr):
        """Enqueues a copy of view v's depth map into device memory at ptr."""
        self.ctx.check(self.ctx._L.rcmvs_scene_depth_to_device(self.ctx.ptr, self.ptr, v, ptr))

    def set_depth(self, v, depth):
        """View v's depth map from a numpy array (copied before return) or a
        device address (copied on the library's stream)."""
        if isinstance(depth, np.ndarray):
            d = np.ascontiguousarray(depth, dtype=np.float32)
            assert d.size == self.views[v].w * self.views[v].h
            self.ctx.check(self.ctx._L.rcmvs_scene_set_depth(self.ctx.ptr, self.ptr, v, d.ctypes.data, 0))
        else:
            self.ctx.check(self.ctx._L.rcmvs_scene_set_depth(self.ctx.ptr, self.ptr, v, int(depth), 1))

    def fuse_candidates_device(self, fusion_order, ref_views, opts):
        """fuse_candidates with the candidates kept on the device; returns
        (count, per-view counts)."""
        off, flat = _csr(fusion_order)
        refs = np.array(list(ref_views) or [0], np.int32)
        per_view = np.zeros(len(self.views), np.uint64)
        n = C.c_uint64()
        o = opts.to_c()
        self.ctx.check(self.ctx._L.rcmvs_scene_fuse_candidates_device(self.ctx.ptr, self.ptr, off.ctypes.data,
                                                                      flat.ctypes.data, refs.ctypes.data,
                                                                      len(ref_views), C.byref(o), C.byref(n),
                                                                      per_view.ctypes.data))
        return n.value, per_view

    def candidates_to_device(self, xyz_ptr, rgb_ptr):
        """Enqueues copies of the kept candidates (n x 3 f64, n x 3 u8)."""
        self.ctx.check(self.ctx._L.rcmvs_scene_candidates_to_device(self.ctx.ptr, self.ptr, xyz_ptr, rgb_ptr))

    def fuse_reduce_device(self, xyz_ptr, rgb_ptr, n, sparse_xyz, opts):
        """Voxel dedup of n device-resident candidates into the scene's cloud
        (read with points()); returns the point count."""
        sp = np.ascontiguousarray(sparse_xyz, dtype=np.float64)
        npts = C.c_uint64()
        o = opts.to_c()
        self.ctx.check(self.ctx._L.rcmvs_scene_fuse_reduce_device(self.ctx.ptr, self.ptr, xyz_ptr, rgb_ptr, int(n),
                                                                  sp.ctypes.data, len(sp), C.byref(o),
                                                                  C.byref(npts)))
        self.n_points = npts.value
        return npts.value

    def depth(self, v, normals=False):
        w, h = self.views[v].w, self.views[v].h
        d = np.empty((h, w), np.float32)
        c = np.empty((h, w), np.float32)
        n = np.empty((h, w, 3), np.float32) if normals else None
        self.ctx.check(self.ctx._L.rcmvs_scene_get_depth(self.ctx.ptr, self.ptr, v, d.ctypes.data, c.ctypes.data,
                                                         _abi.ptr(n)))
        return DepthMap(d, c, n)

    def census(self, v):
        w, h = self.views[v].w, self.views[v].h
        out = np.empty((h, w), np.uint64)
        self.ctx.check(self.ctx._L.rcmvs_scene_get_census(self.ctx.ptr, self.ptr, v, out.ctypes.data))
        return out

    def points(self, ply_body=False):
        n = self.n_points
        xyz = np.empty((n, 3), np.float64)
        rgb = np.empty((n, 3), np.uint8)
        body = np.empty(15 * n, np.uint8) if ply_body else None
        if n:
            self.ctx.check(self.ctx._L.rcmvs_scene_get_points(self.ctx.ptr, self.ptr, xyz.ctypes.data,
                                                              rgb.ctypes.data, _abi.ptr(body)))
        return (xyz, rgb, body) if ply_body else (xyz, rgb)

    def close(self):
        if getattr(self, "ptr", None):
            self.ctx._L.rcmvs_scene_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_dense_outputs(dense_dir, xyz, rgb, stats=None, web_cap=0):
    """The files run_mvs writes (lib.rs:429-501): dense.ply, dense_web.json
    and, with stats (an MvsStats), mvs_stats.json, by the library's writer."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1, 3)
    st = None
    if stats is not None:
        st = _abi.Stats()
        st.views, st.views_with_depth, st.dense_points = stats.views, stats.views_with_depth, stats.dense_points
        st.fusion_candidates = stats.fusion_candidates
        st.elapsed_s, st.stereo_s, st.fuse_s = stats.elapsed_s, stats.stereo_s, stats.fuse_s
    rc = _lib.mvs().rcmvs_write_dense_outputs(os.fsencode(dense_dir), xyz.ctypes.data, rgb.ctypes.data, len(xyz),
                                              C.byref(st) if st is not None else None, int(web_cap))
    if rc != 0:
        raise RcmvsError(rc, f"cannot write the dense outputs into {dense_dir}")


def run_mvs(views, sparse, opts, out_dir=None, ctx=None, log=None, return_depth=False, net=None,
            conf_thr=None, n_local=1, span=0.0):
    """mvs::run_mvs (lib.rs:294-517) from views already at working resolution
    (the image decode/resize of load_views is not part of this path).  Writes
    <out_dir>/dense/dense.ply, mvs_stats.json and dense_web.json when out_dir
    is given.  net (a learned.ProposalNet, extension): seed stereo with the
    network instead of the plane sweep (conf_thr None: the learned module's
    operating point).  Returns (MvsStats, xyz, rgb[, depth maps])."""
    ctx = _ctx(ctx)
    if conf_thr is None:
        from .learned import CONF_THR as conf_thr
    t0 = time.time()
    if len(views) < 2:
        raise RcmvsError(_abi.RCMVS_E_ARG, "need at least 2 registered views for MVS")
    if len(sparse.xyz) < 8:
        raise RcmvsError(_abi.RCMVS_E_ARG,
                         f"sparse reconstruction too small for MVS ({len(sparse.xyz)} points, need >= 8)")
    va = _abi.view_array(views)
    sp = sparse.to_c()
    o = opts.to_c()
    st = _abi.Stats()
    pts = _abi.Points()
    douts = None
    dms = []
    want_vis = bool(opts.save_depth_vis) and out_dir is not None  # lib.rs:383-389
    if return_depth or want_vis:
        douts = (_abi.DepthOut * len(views))()
        for i, v in enumerate(views):
            d = np.empty((v.h, v.w), np.float32)
            c = np.empty((v.h, v.w), np.float32)
            douts[i] = _abi.DepthOut(d.ctypes.data, c.ctypes.data, None)
            dms.append(DepthMap(d, c))
    if net is None:
        ctx.check(ctx._L.rcmvs_run_mvs(ctx.ptr, va, len(views), C.byref(sp), C.byref(o), douts, C.byref(pts),
                                       C.byref(st)))
    else:
        ctx.check(ctx._L.rcmvs_run_mvs_learned(ctx.ptr, va, len(views), C.byref(sp), C.byref(o), net.ptr,
                                               float(conf_thr), int(n_local), float(span), douts, C.byref(pts),
                                               C.byref(st)))
    xyz, rgb = _take_points(ctx, pts)
    if want_vis:
        srcs, _, _ = plan(sparse, views, opts)
        vis_dir = os.path.join(out_dir, "dense", "depth_vis")
        os.makedirs(vis_dir, exist_ok=True)
        for i, v in enumerate(views):
            if srcs[i]:  # views with a depth map
                img, _, _ = depth_vis(dms[i].depth, ctx)
                write_png_gray(os.path.join(vis_dir, f"{_vis_stem(v.name)}_depth.png"), img)
    stats = MvsStats(views=st.views, views_with_depth=st.views_with_depth, dense_points=st.dense_points,
                     per_view_valid=[int((d.depth > 0).sum()) for d in dms] if return_depth else [],
                     elapsed_s=time.time() - t0, stereo_s=st.stereo_s, fuse_s=st.fuse_s,
                     fusion_candidates=st.fusion_candidates)
    if log:
        log(f"mvs: fused {stats.dense_points} dense points from {stats.views_with_depth} depth maps")
    if out_dir is not None:
        dense = os.path.join(out_dir, "dense")
        os.makedirs(dense, exist_ok=True)
        write_dense_outputs(dense, xyz, rgb, stats)
    return (stats, xyz, rgb, dms) if return_depth else (stats, xyz, rgb)


__all__ = ["Context", "default_context", "census_map", "estimate_depth", "estimate_depth_batch",
           "fuse_depth_maps", "write_ply_binary", "write_dense_outputs", "depth_vis", "write_png_gray", "plan", "run_mvs", "plane_cost_field", "DeviceScene",
           "MvsOptions", "MvsStats", "ViewData", "DepthMap", "SparseModel", "RcmvsError"]
