"""Plain data types of the dense stage, mirroring the reference `mvs` crate.

MvsOptions  <- mvs/src/lib.rs:33-70   (same fields, same defaults)
MvsStats    <- mvs/src/lib.rs:72-79
ViewData    <- mvs/src/lib.rs:86-101  (grey kept as u8; census computed on device)
DepthMap    <- mvs/src/stereo.rs:33-38 (+ optional normals, an extension)
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _abi

# RCMVS_FLAG_* bits of MvsOptions.flags (include/rcmvs.h).  The first five
# leave the results bit-identical.
FLAG_ONE_CANDIDATE = 1  # one-candidate-at-a-time init schedule
FLAG_PERSISTENT = 2     # persistent (view, tile) work-queue launches
FLAG_CUDA_GRAPH = 4     # replay the init/pass/gate schedule from a CUDA graph
FLAG_AUTOTUNE = 8       # per-resolution-class tile shapes from the autotuner
FLAG_NO_SKIP_DUPLICATES = 16  # reference call sequence: no duplicate skip, no early rejection (work counts)
FLAG_INIT_ONLY = 32     # diagnostic: init and gate only, no passes
FLAG_SEED_AND_SWEEP = 64  # learned init: seeded pixels also run the plane sweep
FLAG_ROW_STEP_INIT = 128  # row-step plane sweep instead of the default table sweep
FLAG_NO_REPEAT_SKIP = 256  # evaluate unchanged neighbours' planes again (the repeat skip off)
FLAG_LOCKSTEP_PASSES = 512  # passes one thread per pixel in lockstep (not streamed)
FLAGS_BATCHED = FLAG_PERSISTENT | FLAG_CUDA_GRAPH | FLAG_AUTOTUNE


@dataclass
class MvsOptions:
    max_dim: int = 900
    num_sources: int = 3
    sweeps: int = 4
    num_hyp: int = 48
    min_consistent: int = 2
    depth_diff: float = 0.03
    cost_thr: float = 0.38
    voxel_rel: float = 0.0015
    save_depth_vis: bool = False
    # extensions with no reference counterpart
    reproj_px: float = 0.0
    tile_w: int = 0
    tile_h: int = 0
    flags: int = 0  # RCMVS_FLAG_* bits
    threads_per_pixel: int = 0  # Jacobi passes: 0/1 one thread per pixel, 5 five lanes per pixel
    passes: int = 0  # Jacobi passes; 0 = 2 * max(sweeps, 1), the reference's schedule

    def to_c(self) -> _abi.Options:
        o = _abi.Options()
        o.max_dim = self.max_dim
        o.num_sources = self.num_sources
        o.sweeps = self.sweeps
        o.num_hyp = self.num_hyp
        o.min_consistent = self.min_consistent
        o.save_depth_vis = int(bool(self.save_depth_vis))
        o.cost_thr = self.cost_thr
        o.depth_diff = self.depth_diff
        o.voxel_rel = self.voxel_rel
        o.reproj_px = self.reproj_px
        o.tile_w = self.tile_w
        o.tile_h = self.tile_h
        o.flags = self.flags
        o.threads_per_pixel = self.threads_per_pixel
        o.passes = self.passes
        return o


@dataclass
class MvsStats:
    views: int = 0
    views_with_depth: int = 0
    dense_points: int = 0
    per_view_valid: List[int] = field(default_factory=list)
    elapsed_s: float = 0.0
    stereo_s: float = 0.0
    fuse_s: float = 0.0
    fusion_candidates: int = 0


@dataclass
class Cam:
    """SIMPLE_RADIAL camera (sfm-lite/src/geom.rs:14-20)."""

    f: float
    cx: float
    cy: float
    k: float = 0.0

    def __iter__(self):
        return iter((self.f, self.cx, self.cy, self.k))


@dataclass
class ViewData:
    """One view at working resolution.  gray: (h, w) u8; rgb: (h, w, 3) u8;
    R (3, 3), t (3,): world->camera pose."""

    name: str
    image_id: int
    w: int
    h: int
    cam: Cam
    R: np.ndarray
    t: np.ndarray
    gray: np.ndarray
    rgb: Optional[np.ndarray] = None


@dataclass
class DepthMap:
    depth: np.ndarray  # (h, w) f32, 0 = invalid
    cost: np.ndarray  # (h, w) f32
    normal: Optional[np.ndarray] = None  # (h, w, 3) f32, extension


@dataclass
class SparseModel:
    """The part of a COLMAP reconstruction the dense stage reads: point
    positions and, per point, the views that observe it (track)."""

    xyz: np.ndarray  # (n, 3) f64
    track_offsets: np.ndarray  # (n+1,) u64
    track_views: np.ndarray  # (m,) i32

    def to_c(self):
        return _abi.sparse_struct(self.xyz, self.track_offsets, self.track_views)
