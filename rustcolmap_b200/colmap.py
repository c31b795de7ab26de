"""COLMAP sparse models in and out, and the views the dense stage reads.

Restates, for this path:

* colmap-io/src/lib.rs:14-56    camera model table (ids, names, parameter counts)
* colmap-io/src/lib.rs:244-318  binary readers (cameras.bin, images.bin, points3D.bin)
* colmap-io/src/lib.rs:319-386  binary writers
* colmap-io/src/lib.rs:423-575  text writers and readers (the text reader sorts by id)
* colmap-io/src/lib.rs:578-584  read_dir_any (binary preferred)
* mvs/src/lib.rs:103-117        cam_from_rec (any model -> SIMPLE_RADIAL f, cx, cy, k)
* sfm-lite/src/geom.rs:82-96    quat_to_rot
* mvs/src/lib.rs:158-221        load_views, and the sparse points with their tracks

Images: the reference decodes with the `image` crate (any format), resizes
with its Triangle filter when the long side exceeds `max_dim`, and converts
with `to_luma8` / `to_rgb8`.  Here PNG is decoded by a small decoder (8-bit
grey, grey+alpha, RGB, RGBA; every filter type) and other formats (JPEG,
...) by Pillow (read_image).  A view whose working size differs from its
camera's is resized on the GPU (rcmvs_resize_view: the `image` 0.24
Triangle resampler in f32, in the crate's order of operations).  RGB ->
luma follows the `image` 0.24 conversion, (2126 R + 7152 G + 722 B) / 10000
in integers; for grey input it is the identity.  Neither is pinned by
reference outputs (the crate is not vendored).
"""
import math
import os
import struct
import zlib
from dataclasses import dataclass, field
from decimal import Decimal
from typing import List

import numpy as np

from ._lib import RcmvsError
from .types import Cam, MvsOptions, SparseModel, ViewData

# colmap-io/src/lib.rs:18-48
MODELS = [(0, "SIMPLE_PINHOLE", 3), (1, "PINHOLE", 4), (2, "SIMPLE_RADIAL", 4), (3, "RADIAL", 5),
          (4, "OPENCV", 8), (5, "OPENCV_FISHEYE", 8), (6, "FULL_OPENCV", 12), (7, "FOV", 5),
          (8, "SIMPLE_RADIAL_FISHEYE", 4), (9, "RADIAL_FISHEYE", 5), (10, "THIN_PRISM_FISHEYE", 12)]
_BY_ID = {m[0]: m for m in MODELS}
_BY_NAME = {m[1]: m for m in MODELS}
SIMPLE_PINHOLE, PINHOLE, SIMPLE_RADIAL, RADIAL, OPENCV = 0, 1, 2, 3, 4


@dataclass
class Camera:
    camera_id: int
    model_id: int
    width: int
    height: int
    params: List[float]


@dataclass
class Image:
    """World->camera pose: x_cam = R(qvec) x_world + tvec; qvec = (qw, qx, qy, qz)."""
    image_id: int
    qvec: List[float]
    tvec: List[float]
    camera_id: int
    name: str
    xys: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.float64))
    point3d_ids: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))


@dataclass
class Point3D:
    point3d_id: int
    xyz: List[float]
    rgb: List[int]
    error: float
    track: List[tuple]  # (image_id, point2d_idx)


@dataclass
class Reconstruction:
    cameras: List[Camera] = field(default_factory=list)
    images: List[Image] = field(default_factory=list)
    points3d: List[Point3D] = field(default_factory=list)

    def camera(self, cid):
        for c in self.cameras:
            if c.camera_id == cid:
                return c
        return None

    def sort_all(self):
        self.cameras.sort(key=lambda c: c.camera_id)
        self.images.sort(key=lambda i: i.image_id)
        self.points3d.sort(key=lambda p: p.point3d_id)


def _model(mid):
    if mid not in _BY_ID:
        raise RcmvsError(-1, f"unknown camera model id {mid}")
    return _BY_ID[mid]


# ------------------------------------------------------------------ binary
class _Reader:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.b = f.read()
        self.o = 0
        self.path = path

    def take(self, fmt):
        n = struct.calcsize(fmt)
        if self.o + n > len(self.b):
            raise RcmvsError(-5, f"{self.path}: unexpected end of file")
        v = struct.unpack_from(fmt, self.b, self.o)
        self.o += n
        return v

    def array(self, dtype, count):
        n = np.dtype(dtype).itemsize * count
        if self.o + n > len(self.b):
            raise RcmvsError(-5, f"{self.path}: unexpected end of file")
        a = np.frombuffer(self.b, dtype=dtype, count=count, offset=self.o).copy()
        self.o += n
        return a


def read_cameras_bin(path):
    r = _Reader(path)
    (n,) = r.take("<Q")
    out = []
    for _ in range(n):
        cid, mid, w, h = r.take("<iiQQ")
        npar = _model(mid)[2]
        out.append(Camera(cid, mid, w, h, list(r.take(f"<{npar}d"))))
    return out


def read_images_bin(path):
    r = _Reader(path)
    (n,) = r.take("<Q")
    out = []
    for _ in range(n):
        (iid,) = r.take("<i")
        q = list(r.take("<4d"))
        t = list(r.take("<3d"))
        (cid, ln) = r.take("<iB")
        name = bytes(r.take(f"<{ln}s")[0]).decode("utf-8")
        (npt,) = r.take("<Q")
        rec = r.array(np.dtype([("x", "<f8"), ("y", "<f8"), ("id", "<i8")]), npt)
        out.append(Image(iid, q, t, cid, name, np.stack([rec["x"], rec["y"]], 1).reshape(-1, 2),
                         rec["id"].astype(np.int64)))
    return out


def read_points3d_bin(path):
    r = _Reader(path)
    (n,) = r.take("<Q")
    out = []
    for _ in range(n):
        pid, x, y, z, cr, cg, cb, err, tl = r.take("<qdddBBBdQ")
        tr = r.array(np.dtype([("img", "<i4"), ("idx", "<i4")]), tl)
        out.append(Point3D(pid, [x, y, z], [cr, cg, cb], err,
                           [(int(a), int(b) & 0xFFFFFFFF) for a, b in zip(tr["img"], tr["idx"])]))
    return out


def write_bin_dir(rec, d):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "cameras.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(rec.cameras)))
        for c in rec.cameras:
            f.write(struct.pack("<iiQQ", c.camera_id, c.model_id, c.width, c.height))
            f.write(struct.pack(f"<{len(c.params)}d", *c.params))
    with open(os.path.join(d, "images.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(rec.images)))
        for im in rec.images:
            nb = im.name.encode("utf-8")
            if len(nb) > 255:
                raise RcmvsError(-1, f"image name longer than 255 bytes: {len(nb)}")
            f.write(struct.pack("<i4d3diB", im.image_id, *im.qvec, *im.tvec, im.camera_id, len(nb)) + nb)
            f.write(struct.pack("<Q", len(im.point3d_ids)))
            rec2 = np.zeros(len(im.point3d_ids), np.dtype([("x", "<f8"), ("y", "<f8"), ("id", "<i8")]))
            if len(rec2):
                rec2["x"], rec2["y"], rec2["id"] = im.xys[:, 0], im.xys[:, 1], im.point3d_ids
            f.write(rec2.tobytes())
    with open(os.path.join(d, "points3D.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(rec.points3d)))
        for p in rec.points3d:
            f.write(struct.pack("<qdddBBBdQ", p.point3d_id, *p.xyz, *p.rgb, p.error, len(p.track)))
            for a, b in p.track:
                f.write(struct.pack("<iI", a, b))  # the index's i32 bits, read back `as u32`


def read_bin_dir(d):
    return Reconstruction(read_cameras_bin(os.path.join(d, "cameras.bin")),
                          read_images_bin(os.path.join(d, "images.bin")),
                          read_points3d_bin(os.path.join(d, "points3D.bin")))


# ------------------------------------------------------------------ text
def _rust_f64(x):
    """Rust's `{}` for f64: shortest round-trip digits, never an exponent."""
    x = float(x)
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "inf" if x > 0 else "-inf"
    return format(Decimal(repr(x)).normalize(), "f")


def write_txt_dir(rec, d):
    os.makedirs(d, exist_ok=True)
    s = ["# Camera list with one line of data per camera:\n",
         "#   CAMERA_ID, MODEL, WIDTH, HEIGHT, PARAMS[]\n",
         "# Supported models: " + ", ".join(m[1] for m in MODELS) + "\n"]
    for c in rec.cameras:
        name = _BY_ID[c.model_id][1] if c.model_id in _BY_ID else "UNKNOWN"
        s.append(f"{c.camera_id} {name} {c.width} {c.height}" + "".join(" " + _rust_f64(p) for p in c.params)
                 + "\n")
    with open(os.path.join(d, "cameras.txt"), "w") as f:
        f.write("".join(s))
    s = ["# Image list with two lines of data per image:\n",
         "#   IMAGE_ID, QW, QX, QY, QZ, TX, TY, TZ, CAMERA_ID, NAME\n",
         "#   POINTS2D[] as (X, Y, POINT3D_ID)\n"]
    for im in rec.images:
        s.append(" ".join([str(im.image_id)] + [_rust_f64(v) for v in list(im.qvec) + list(im.tvec)] +
                          [str(im.camera_id), im.name]) + "\n")
        s.append(" ".join(f"{_rust_f64(x)} {_rust_f64(y)} {int(i)}"
                          for (x, y), i in zip(im.xys, im.point3d_ids)) + "\n")
    with open(os.path.join(d, "images.txt"), "w") as f:
        f.write("".join(s))
    s = ["# 3D point list with one line of data per point:\n",
         "#   POINT3D_ID, X, Y, Z, R, G, B, ERROR, TRACK[] as (IMAGE_ID, POINT2D_IDX)\n"]
    for p in rec.points3d:
        s.append(" ".join([str(p.point3d_id)] + [_rust_f64(v) for v in p.xyz] + [str(v) for v in p.rgb] +
                          [_rust_f64(p.error)]) + "".join(f" {a} {b}" for a, b in p.track) + "\n")
    with open(os.path.join(d, "points3D.txt"), "w") as f:
        f.write("".join(s))


def _data_lines(path):
    with open(path) as f:
        return [l.rstrip("\n") for l in f if not l.lstrip().startswith("#")]


def _f64(s):
    try:
        return float(s)
    except ValueError:
        raise RcmvsError(-5, f"bad float `{s}`")


def _i64(s):
    try:
        return int(s)
    except ValueError:
        raise RcmvsError(-5, f"bad int `{s}`")


def read_txt_dir(d):
    cams = []
    for line in _data_lines(os.path.join(d, "cameras.txt")):
        t = line.split()
        if len(t) < 5:
            continue
        m = _BY_NAME.get(t[1].upper())
        if m is None:
            raise RcmvsError(-5, f"unknown model `{t[1]}`")
        cams.append(Camera(_i64(t[0]), m[0], _i64(t[2]), _i64(t[3]), [_f64(v) for v in t[4:4 + m[2]]]))
    images = []
    lines = _data_lines(os.path.join(d, "images.txt"))
    for k in range(0, len(lines), 2):
        t = lines[k].split()
        l2 = lines[k + 1] if k + 1 < len(lines) else ""
        if len(t) < 10:
            continue
        toks = l2.split()
        trip = [toks[i:i + 3] for i in range(0, len(toks), 3) if len(toks[i:i + 3]) == 3]
        xys = np.array([[_f64(a), _f64(b)] for a, b, _ in trip], np.float64).reshape(-1, 2)
        ids = np.array([_i64(c) for _, _, c in trip], np.int64)
        images.append(Image(_i64(t[0]), [_f64(v) for v in t[1:5]], [_f64(v) for v in t[5:8]], _i64(t[8]),
                            " ".join(t[9:]), xys, ids))
    pts = []
    for line in _data_lines(os.path.join(d, "points3D.txt")):
        t = line.split()
        if len(t) < 8:
            continue
        tr = [(_i64(t[i]), _i64(t[i + 1]) & 0xFFFFFFFF) for i in range(8, len(t) - 1, 2)]
        pts.append(Point3D(_i64(t[0]), [_f64(v) for v in t[1:4]], [_i64(v) & 0xFF for v in t[4:7]], _f64(t[7]),
                           tr))
    rec = Reconstruction(cams, images, pts)
    rec.sort_all()
    return rec


def read_dir_any(d):
    """Binary if cameras.bin exists, else text (colmap-io/src/lib.rs:578-584)."""
    return read_bin_dir(d) if os.path.exists(os.path.join(d, "cameras.bin")) else read_txt_dir(d)


# ------------------------------------------------------------------ geometry
def quat_to_rot(q):
    """sfm-lite/src/geom.rs:82-96, f64 in the same operation order."""
    w, x, y, z = (float(v) for v in q)
    n = w * w + x * x + y * y + z * z
    if abs(n) - 1.0 > 1e-12:
        s = np.sqrt(n)
        w, x, y, z = w / s, x / s, y / s, z / s
    return np.array([[1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - w * z), 2.0 * (x * z + w * y)],
                     [2.0 * (x * y + w * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - w * x)],
                     [2.0 * (x * z - w * y), 2.0 * (y * z + w * x), 1.0 - 2.0 * (x * x + y * y)]], np.float64)


def cam_from_rec(c, sx, sy):
    """mvs/src/lib.rs:103-117: SIMPLE_RADIAL (f, cx, cy, k) of any model;
    models other than SIMPLE_RADIAL get k = 0."""
    p = c.params

    def g(i):
        return float(p[i]) if i < len(p) else 0.0
    if c.model_id == SIMPLE_PINHOLE:
        f, cx, cy, k = g(0), g(1), g(2), 0.0
    elif c.model_id == SIMPLE_RADIAL:
        f, cx, cy, k = g(0), g(1), g(2), g(3)
    elif c.model_id == RADIAL:
        f, cx, cy, k = g(0), g(2), g(3), 0.0
    elif c.model_id in (PINHOLE, OPENCV):
        f, cx, cy, k = 0.5 * (g(0) + g(1)), g(2), g(3), 0.0
    else:
        f, cx, cy, k = g(0), g(2), g(3), 0.0
    s = 0.5 * (sx + sy)
    return Cam(f * s, cx * sx, cy * sy, k)


def _round_half_away(x):
    """f64::round for x >= 0 (Python's round() goes half to even)."""
    f = math.floor(x)
    return int(f) + (1 if x - f >= 0.5 else 0)


def working_size(width, height, max_dim):
    """mvs/src/lib.rs:155-157, :185-187."""
    s = min(float(max_dim) / float(max(width, height)), 1.0)
    return max(_round_half_away(width * s), 16), max(_round_half_away(height * s), 16)


# ------------------------------------------------------------------ images
def read_png(path):
    """8-bit PNG (grey, grey+alpha, RGB, RGBA; any filter; no interlace) ->
    (h, w, channels) u8."""
    with open(path, "rb") as f:
        b = f.read()
    if b[:8] != b"\x89PNG\r\n\x1a\n":
        raise RcmvsError(-5, f"{path}: not a PNG file (only PNG is decoded here)")
    pos, idat, hdr = 8, [], None
    while pos + 8 <= len(b):
        (n,) = struct.unpack(">I", b[pos:pos + 4])
        typ, data = b[pos + 4:pos + 8], b[pos + 8:pos + 8 + n]
        if typ == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", data)
        elif typ == b"IDAT":
            idat.append(data)
        elif typ == b"IEND":
            break
        pos += 12 + n
    if hdr is None:
        raise RcmvsError(-5, f"{path}: no IHDR")
    w, h, depth, ctype, _, _, inter = hdr
    chans = {0: 1, 4: 2, 2: 3, 6: 4}.get(ctype)
    if depth != 8 or chans is None or inter != 0:
        raise RcmvsError(-5, f"{path}: only 8-bit non-interlaced grey/RGB(A) PNG is supported")
    raw = np.frombuffer(zlib.decompress(b"".join(idat)), np.uint8)
    stride = w * chans
    raw = raw[:h * (stride + 1)].reshape(h, stride + 1)
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros((w, chans), np.int32)
    for y in range(h):
        ft, line = raw[y, 0], raw[y, 1:].astype(np.int32).reshape(w, chans)
        if ft == 0:  # None
            cur = line
        elif ft == 1:  # Sub: running sum along the row, per channel
            cur = np.cumsum(line, axis=0) & 0xFF
        elif ft == 2:  # Up
            cur = (line + prev) & 0xFF
        elif ft in (3, 4):  # Average / Paeth: pixel by pixel
            cur = np.zeros((w, chans), np.int32)
            a = np.zeros(chans, np.int32)
            c = np.zeros(chans, np.int32)
            for i in range(w):
                bb = prev[i]
                if ft == 3:
                    pr = (a + bb) >> 1
                else:
                    p0 = a + bb - c
                    pa, pb, pc = np.abs(p0 - a), np.abs(p0 - bb), np.abs(p0 - c)
                    pr = np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, bb, c))
                cur[i] = (line[i] + pr) & 0xFF
                a, c = cur[i], bb
        else:
            raise RcmvsError(-5, f"{path}: bad PNG filter {ft}")
        out[y] = cur.reshape(-1)
        prev = cur
    return out.reshape(h, w, chans)


def _png_with_pillow(path):
    """An 8-bit grey/RGB(A) PNG decoded by Pillow (PNG is lossless, so the
    pixels are read_png's), or None when Pillow is missing or the file holds
    another kind of PNG."""
    try:
        from PIL import Image
    except ImportError:
        return None
    try:
        with Image.open(path) as im:
            if im.format != "PNG" or im.mode not in ("L", "LA", "RGB", "RGBA") or im.info.get("interlace"):
                return None
            a = np.asarray(im, dtype=np.uint8)
    except OSError:
        return None
    return np.ascontiguousarray(a.reshape(a.shape[0], a.shape[1], -1))


def read_image(path):
    """Decoded 8-bit image (h, w, channels).  PNG gives the pixels the
    reference's decoder gives: through Pillow when it is installed (its
    per-row filters run in C), else through read_png; other formats (JPEG,
    BMP, TIFF, ...) through Pillow, whose JPEG inverse DCT is not the `image`
    crate's, so lossy images may differ from the reference's by a grey level
    in places.  Palette, 16-bit and other modes are converted to RGB."""
    with open(path, "rb") as f:
        sig = f.read(8)
    if sig == b"\x89PNG\r\n\x1a\n":
        a = _png_with_pillow(path)
        return read_png(path) if a is None else a
    try:
        from PIL import Image
    except ImportError:
        raise RcmvsError(-5, f"{path}: not a PNG and Pillow is not installed to decode it")
    try:
        with Image.open(path) as im:
            mode = im.mode
            if mode not in ("L", "LA", "RGB", "RGBA"):
                im = im.convert("RGB")
                mode = "RGB"
            a = np.asarray(im, dtype=np.uint8)
    except OSError as e:
        raise RcmvsError(-5, f"cannot decode {path}: {e}")
    return np.ascontiguousarray(a.reshape(a.shape[0], a.shape[1], -1))


def gray_rgb(img):
    """`to_luma8` / `to_rgb8` of a decoded image: grey as is, RGB -> luma
    (2126 R + 7152 G + 722 B) / 10000 (integer), alpha dropped."""
    c = img.shape[2]
    if c in (1, 2):
        g = img[:, :, 0].copy()
        return g, np.repeat(g[:, :, None], 3, axis=2)
    rgb = np.ascontiguousarray(img[:, :, :3])
    r, gg, b = (rgb[:, :, i].astype(np.uint32) for i in range(3))
    return ((2126 * r + 7152 * gg + 722 * b) // 10000).astype(np.uint8), rgb


def load_views(rec, image_dir, opts=None, ctx=None):
    """mvs/src/lib.rs:158-221 (views in rec.images order) plus the sparse
    points with tracks as view indices (entries of unknown images dropped,
    as lib.rs:227-231 skips them).  Images whose camera is larger than
    max_dim are resized on the GPU of `ctx` (the default context when None).
    Returns (views, SparseModel)."""
    opts = opts or MvsOptions()
    views = []
    for im in rec.images:
        c = rec.camera(im.camera_id)
        if c is None:
            raise RcmvsError(-1, f"image {im.name} references missing camera {im.camera_id}")
        mw, mh = working_size(c.width, c.height, opts.max_dim)
        cam = cam_from_rec(c, mw / c.width, mh / c.height)
        path = os.path.join(image_dir, im.name)
        try:
            img = read_image(path)
        except OSError as e:
            raise RcmvsError(-5, f"cannot open {path}: {e}")
        if (mw, mh) != (c.width, c.height):  # lib.rs:188-190
            from . import mvs
            g, rgb = mvs.resize_view(img, mw, mh, ctx)
        else:
            g, rgb = gray_rgb(img)
        views.append(ViewData(im.name, im.image_id, g.shape[1], g.shape[0], cam, quat_to_rot(im.qvec),
                              np.array(im.tvec, np.float64), g, rgb))
    if len(views) < 2:
        raise RcmvsError(-1, "need at least 2 registered views for MVS")
    idx = {im.image_id: i for i, im in enumerate(rec.images)}
    xyz = np.array([p.xyz for p in rec.points3d], np.float64).reshape(-1, 3)
    off = np.zeros(len(rec.points3d) + 1, np.uint64)
    tv = []
    for k, p in enumerate(rec.points3d):
        tv.extend(idx.get(a, -1) for a, _ in p.track)
        off[k + 1] = len(tv)
    return views, SparseModel(xyz, off, np.array(tv, np.int32))


def run_mvs_colmap(sparse_dir, image_dir, out_dir, opts=None, ctx=None, net=None, log=None):
    """mvs::run_mvs (mvs/src/lib.rs:294-300) from a COLMAP model (a model
    directory or a Reconstruction, as the reference takes) and its images:
    load_views, stereo, fusion, and the files under <out_dir>/dense.
    Returns (MvsStats, xyz, rgb)."""
    from . import mvs
    opts = opts or MvsOptions()
    rec = sparse_dir if isinstance(sparse_dir, Reconstruction) else read_dir_any(sparse_dir)
    views, sparse = load_views(rec, image_dir, opts, ctx)
    if log:
        log(f"mvs: loaded {len(views)} views at working resolution (max_dim {opts.max_dim})")
    return mvs.run_mvs(views, sparse, opts, out_dir=out_dir, ctx=ctx, log=log, net=net)
