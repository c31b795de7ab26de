"""SIFT features and descriptor matching on the GPU: the mirrors of
`sift::extract_sift` (sfm-lite/src/sift.rs:435-555) and
`matching::match_pair` (sfm-lite/src/matching.rs:22-95) over librcmvs
(rcmvs_extract_sift, rcmvs_match_pairs).

There is no CPU path: a missing library or a CUDA error raises RcmvsError.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._lib import RcmvsError  # noqa: F401

DESC_LEN = 128


@dataclass
class SiftOptions:
    """`sift::SiftOptions` (sift.rs:20-32) with its defaults."""
    max_dim: int = 1600
    max_features: int = 2048
    contrast_thr: float = 0.0067

    def to_c(self):
        return _abi.SiftOptions(self.max_dim, self.max_features, 0, 0, self.contrast_thr)


@dataclass
class SiftFrame:
    """`sift::SiftFrame` (sift.rs:34-41)."""
    name: str
    width: int
    height: int
    pts: np.ndarray                      # (n, 2) f64
    desc: np.ndarray                     # (n, 128) f32
    colors: np.ndarray                   # (n, 3) u8
    n_raw: int = 0                       # extrema kept by the fit (diagnostic)
    extra: dict = field(default_factory=dict)


def extract_sift(img, name="", opts=None, ctx=None):
    """SIFT keypoints and descriptors of one decoded 8-bit image ((h, w) or
    (h, w, c), c = 1-4) on the GPU."""
    from .mvs import _ctx
    ctx = _ctx(ctx)
    opts = opts or SiftOptions()
    a = np.ascontiguousarray(img, dtype=np.uint8)
    if a.ndim == 2:
        a = a[:, :, None]
    h, w, c = a.shape
    o = opts.to_c()
    f = _abi.SiftFrame()
    ctx.check(ctx._L.rcmvs_extract_sift(ctx.ptr, a.ctypes.data, w, h, c, C.byref(o), C.byref(f)))
    try:
        n = f.n
        k = max(n, 1)
        pts = np.ctypeslib.as_array((C.c_double * (2 * k)).from_address(f.pts))[: 2 * n].reshape(n, 2).copy()
        desc = np.ctypeslib.as_array((C.c_float * (DESC_LEN * k)).from_address(f.desc))[: DESC_LEN * n]
        desc = desc.reshape(n, DESC_LEN).copy()
        col = np.ctypeslib.as_array((C.c_uint8 * (3 * k)).from_address(f.colors))[: 3 * n].reshape(n, 3).copy()
        return SiftFrame(name, f.width, f.height, pts, desc, col, int(f.n_raw))
    finally:
        ctx._L.rcmvs_sift_frame_free(C.byref(f))


def extract_sift_many(images, names=None, opts=None, ctxs=None):
    """extract_sift of every image, spread over the contexts `ctxs` (one
    CUDA stream each) with one host thread per context: an extraction waits
    on its stream a few times per image (keypoint counts, chunked
    descriptors, results) and the library call releases the GIL, so the
    images' round trips and kernels overlap.  Image i runs on context
    i % len(ctxs); each result is the single-context one (same kernels, same
    order of operations per image).  Returns the frames in image order."""
    from concurrent.futures import ThreadPoolExecutor

    from .mvs import _ctx
    ctxs = list(ctxs) if ctxs else [_ctx(None)]
    names = names or [""] * len(images)
    nw = len(ctxs)
    if nw == 1 or len(images) < 2:
        return [extract_sift(im, nm, opts, ctxs[0]) for im, nm in zip(images, names)]

    def share(w):
        return [(i, extract_sift(images[i], names[i], opts, ctxs[w])) for i in range(w, len(images), nw)]

    frames = [None] * len(images)
    with ThreadPoolExecutor(nw) as ex:
        for part in ex.map(share, range(nw)):
            for i, f in part:
                frames[i] = f
    return frames


def match_pairs(descs, pairs, ratio=0.8, ctx=None):
    """match_pair for many pairs of frames in one batched call.  descs: list
    of (n_f, 128) f32 descriptor arrays; pairs: list of (i, j).  Returns one
    (a indices, b indices) pair of u32 arrays per pair, in the reference's
    order."""
    from .mvs import _ctx
    ctx = _ctx(ctx)
    ds = [np.ascontiguousarray(d, dtype=np.float32).reshape(-1, DESC_LEN) for d in descs]
    ptrs = (C.c_void_p * max(len(ds), 1))(*[d.ctypes.data if len(d) else None for d in ds])
    nd = np.array([len(d) for d in ds] or [0], np.int32)
    pr = np.array(list(pairs) or [(0, 0)], np.int32).reshape(-1, 2)
    m = _abi.Matches()
    ctx.check(ctx._L.rcmvs_match_pairs(ctx.ptr, ptrs, nd.ctypes.data, len(ds), pr.ctypes.data, len(pairs),
                                       float(ratio), C.byref(m)))
    try:
        npairs = len(pairs)
        off = np.ctypeslib.as_array((C.c_uint64 * (npairs + 1)).from_address(m.offsets)).copy()
        tot = int(off[-1])
        k = max(tot, 1)
        a = np.ctypeslib.as_array((C.c_uint32 * k).from_address(m.a))[:tot].copy()
        b = np.ctypeslib.as_array((C.c_uint32 * k).from_address(m.b))[:tot].copy()
        return [(a[off[p]:off[p + 1]], b[off[p]:off[p + 1]]) for p in range(npairs)]
    finally:
        ctx._L.rcmvs_matches_free(C.byref(m))


def match_pair(fa, fb, ratio=0.8, ctx=None):
    """matching::match_pair of two SiftFrames (or descriptor arrays)."""
    da = fa.desc if isinstance(fa, SiftFrame) else fa
    db = fb.desc if isinstance(fb, SiftFrame) else fb
    return match_pairs([da, db], [(0, 1)], ratio, ctx)[0]


def job_pairs(n, sequential=False):
    """The image pairs sfm-lite matches (sfm-lite/src/lib.rs:197-212): each
    image with the next three when `sequential`, else every pair i < j, in
    the reference's order."""
    if sequential:
        return [(i, i + k) for i in range(n) for k in (1, 2, 3) if i + k < n]
    return [(i, j) for i in range(n) for j in range(i + 1, n)]


def extract_and_match(images, names=None, opts=None, ratio=0.75, sequential=False, ctx=None, workers=4):
    """The feature stage of sfm-lite's run_sfm (sfm-lite/src/lib.rs:137-225,
    two-view verification excluded): SIFT of every decoded image (spread
    over `workers` contexts on ctx's device, extract_sift_many), then
    match_pair on every job pair in one batched call on ctx.  `ratio`
    defaults to sfm-lite's Options::default() (lib.rs:61).  Returns (frames,
    pairs, matches) with matches[p] = (a indices, b indices) of pairs[p]."""
    from .mvs import Context, _ctx
    if len(images) < 2:
        raise RcmvsError(-1, "need at least 2 images")
    ctx = _ctx(ctx)
    names = names or [""] * len(images)
    extra = [Context(ctx.device) for _ in range(max(1, min(workers, len(images))) - 1)]
    try:
        frames = extract_sift_many(images, names, opts, [ctx] + extra)
    finally:
        for c in extra:
            c.close()
    pairs = job_pairs(len(frames), sequential)
    return frames, pairs, match_pairs([f.desc for f in frames], pairs, ratio, ctx)


IMAGE_EXTENSIONS = ("jpg", "jpeg", "png", "bmp", "tif", "tiff", "webp")  # sfm-lite/src/lib.rs:83-91


def image_files(images_dir):
    """The images sfm-lite's run_sfm_dir takes (sfm-lite/src/lib.rs:119-126):
    regular files with an image extension (case-insensitive), sorted by
    path."""
    import os
    out = []
    for e in os.listdir(images_dir):
        p = os.path.join(images_dir, e)
        ext = os.path.splitext(e)[1][1:].lower()
        if os.path.isfile(p) and ext in IMAGE_EXTENSIONS:
            out.append(p)
    return sorted(out)


def extract_and_match_dir(images_dir, opts=None, ratio=0.75, sequential=False, ctx=None):
    """extract_and_match over the images of a directory, in run_sfm_dir's
    order; frame names are the file names (sfm-lite/src/lib.rs:141-146)."""
    import os
    from .colmap import read_image
    paths = image_files(images_dir)
    return extract_and_match([read_image(p) for p in paths], [os.path.basename(p) for p in paths], opts, ratio,
                             sequential, ctx)
