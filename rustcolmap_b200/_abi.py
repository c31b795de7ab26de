"""ctypes mirror of the C ABI structs declared in include/rcmvs.h.

Only layouts live here; loading the CUDA library is rustcolmap_b200._lib's job.
"""
import ctypes as C

import numpy as np

RCMVS_OK = 0
RCMVS_E_ARG = -1
RCMVS_E_CUDA = -2
RCMVS_E_NOMEM = -3
RCMVS_E_LIMIT = -4
RCMVS_E_IO = -5
RCMVS_E_STATE = -6
RCMVS_MAX_SOURCES = 32


class Options(C.Structure):
    """rcmvs_options — mirrors mvs::MvsOptions (mvs/src/lib.rs:33-54)."""

    _fields_ = [
        ("max_dim", C.c_uint32),
        ("num_sources", C.c_uint32),
        ("sweeps", C.c_uint32),
        ("num_hyp", C.c_uint32),
        ("min_consistent", C.c_uint32),
        ("save_depth_vis", C.c_uint32),
        ("cost_thr", C.c_float),
        ("passes", C.c_uint32),
        ("depth_diff", C.c_double),
        ("voxel_rel", C.c_double),
        ("reproj_px", C.c_double),
        ("tile_w", C.c_uint32),
        ("tile_h", C.c_uint32),
        ("flags", C.c_uint32),
        ("threads_per_pixel", C.c_uint32),
    ]


class View(C.Structure):
    _fields_ = [
        ("w", C.c_int32),
        ("h", C.c_int32),
        ("f", C.c_double),
        ("cx", C.c_double),
        ("cy", C.c_double),
        ("k", C.c_double),
        ("R", C.c_double * 9),
        ("t", C.c_double * 3),
        ("gray", C.c_void_p),
        ("rgb", C.c_void_p),
    ]


class Job(C.Structure):
    _fields_ = [
        ("ref_idx", C.c_int32),
        ("n_src", C.c_int32),
        ("srcs", C.c_void_p),
        ("zmin", C.c_double),
        ("zmax", C.c_double),
    ]


class TuneEntry(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("tile_w", C.c_int32), ("tile_h", C.c_int32),
                ("threads_per_pixel", C.c_int32), ("reserved", C.c_int32), ("ms_best", C.c_float),
                ("ms_default", C.c_float)]


class SiftOptions(C.Structure):
    _fields_ = [("max_dim", C.c_uint32), ("max_features", C.c_uint32), ("reserved", C.c_uint32),
                ("reserved2", C.c_uint32), ("contrast_thr", C.c_double)]


class SiftFrame(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("n", C.c_uint64), ("n_raw", C.c_uint64),
                ("pts", C.c_void_p), ("desc", C.c_void_p), ("colors", C.c_void_p)]


class Matches(C.Structure):
    _fields_ = [("n_pairs", C.c_uint64), ("offsets", C.c_void_p), ("a", C.c_void_p), ("b", C.c_void_p)]


class DepthOut(C.Structure):
    _fields_ = [("depth", C.c_void_p), ("cost", C.c_void_p), ("normal", C.c_void_p)]


class Sparse(C.Structure):
    _fields_ = [
        ("n_points", C.c_uint64),
        ("xyz", C.c_void_p),
        ("track_offsets", C.c_void_p),
        ("track_views", C.c_void_p),
    ]


class Points(C.Structure):
    _fields_ = [("n", C.c_uint64), ("xyz", C.c_void_p), ("rgb", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [
        ("views", C.c_uint64),
        ("views_with_depth", C.c_uint64),
        ("dense_points", C.c_uint64),
        ("fusion_candidates", C.c_uint64),
        ("elapsed_s", C.c_float),
        ("stereo_s", C.c_float),
        ("fuse_s", C.c_float),
        ("reserved0", C.c_uint32),
    ]


def ptr(a):
    """Data pointer of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], "need a C-contiguous array"
    return a.ctypes.data


def view_array(views):
    """Build a ctypes rcmvs_view[] from objects with w, h, cam (f, cx, cy, k),
    R (3x3), t (3,), gray (h, w) u8 and optional rgb (h, w, 3) u8.  The
    returned array keeps references to the numpy buffers it points at."""
    arr = (View * len(views))()
    keep = []
    for i, v in enumerate(views):
        gray = np.ascontiguousarray(v.gray, dtype=np.uint8)
        rgb = None if getattr(v, "rgb", None) is None else np.ascontiguousarray(v.rgb, dtype=np.uint8)
        keep += [gray, rgb]
        a = arr[i]
        a.w, a.h = int(v.w), int(v.h)
        a.f, a.cx, a.cy, a.k = (float(c) for c in v.cam)
        for j, x in enumerate(np.asarray(v.R, dtype=np.float64).reshape(9)):
            a.R[j] = float(x)
        for j, x in enumerate(np.asarray(v.t, dtype=np.float64).reshape(3)):
            a.t[j] = float(x)
        a.gray = gray.ctypes.data
        a.rgb = None if rgb is None else rgb.ctypes.data
    arr._keep = keep
    return arr


def sparse_struct(xyz, track_offsets, track_views):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    off = np.ascontiguousarray(track_offsets, dtype=np.uint64)
    tv = np.ascontiguousarray(track_views, dtype=np.int32)
    s = Sparse(len(xyz), xyz.ctypes.data, off.ctypes.data, tv.ctypes.data)
    s._keep = (xyz, off, tv)
    return s
