"""COLMAP model IO and view loading (rustcolmap_b200.colmap) against the
reference's colmap-io / load_views semantics: byte layouts, round trips, the
text reader's quirks, camera conversion, quaternions, PNG decoding, and an
end-to-end load of a written model."""
import os
import struct
import zlib

import numpy as np
import pytest

from rustcolmap_b200 import MvsOptions, colmap, mvs, scene
from rustcolmap_b200._lib import RcmvsError


def rot_to_quat(R):
    """Test helper: rotation matrix -> (qw, qx, qy, qz)."""
    tr = R[0, 0] + R[1, 1] + R[2, 2]
    if tr > 0:
        s = np.sqrt(1.0 + tr) * 2
        return [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    i = int(np.argmax(np.diag(R)))
    j, k = (i + 1) % 3, (i + 2) % 3
    s = np.sqrt(1.0 + R[i, i] - R[j, j] - R[k, k]) * 2
    q = [0.0] * 4
    q[0] = (R[k, j] - R[j, k]) / s
    q[1 + i] = 0.25 * s
    q[1 + j] = (R[j, i] + R[i, j]) / s
    q[1 + k] = (R[k, i] + R[i, k]) / s
    return q


def random_rec(seed=0):
    rng = np.random.default_rng(seed)
    cams = [colmap.Camera(3, colmap.SIMPLE_RADIAL, 640, 480, [500.0, 320.5, 240.25, -0.01]),
            colmap.Camera(1, colmap.OPENCV, 1920, 1080, list(rng.normal(size=8)))]
    imgs = []
    for k, name in enumerate(["a.png", "dir/b c.png", "ü.png"]):
        n = int(rng.integers(0, 5))
        imgs.append(colmap.Image(10 - k, list(rng.normal(size=4)), list(rng.normal(size=3)), [3, 1][k % 2], name,
                                 rng.normal(size=(n, 2)), rng.integers(-1, 100, n).astype(np.int64)))
    pts = [colmap.Point3D(int(i), list(rng.normal(size=3)), [int(v) for v in rng.integers(0, 256, 3)],
                          float(rng.uniform()), [(int(a), int(b)) for a, b in zip(rng.integers(0, 12, 3),
                                                                                rng.integers(0, 2**32 - 1, 3))])
           for i in (7, 2, 5)]
    return colmap.Reconstruction(cams, imgs, pts)


def assert_rec_equal(a, b):
    assert [(c.camera_id, c.model_id, c.width, c.height, list(c.params)) for c in a.cameras] == \
        [(c.camera_id, c.model_id, c.width, c.height, list(c.params)) for c in b.cameras]
    assert len(a.images) == len(b.images)
    for x, y in zip(a.images, b.images):
        assert (x.image_id, list(x.qvec), list(x.tvec), x.camera_id, x.name) == \
            (y.image_id, list(y.qvec), list(y.tvec), y.camera_id, y.name)
        assert np.array_equal(x.xys, y.xys) and np.array_equal(x.point3d_ids, y.point3d_ids)
    assert [(p.point3d_id, list(p.xyz), list(p.rgb), p.error, list(p.track)) for p in a.points3d] == \
        [(p.point3d_id, list(p.xyz), list(p.rgb), p.error, list(p.track)) for p in b.points3d]


def test_cameras_bin_byte_layout(tmp_path):
    rec = colmap.Reconstruction([colmap.Camera(4, colmap.SIMPLE_RADIAL, 640, 480, [1.0, 2.0, 3.0, 4.0])], [], [])
    colmap.write_bin_dir(rec, str(tmp_path))
    b = open(tmp_path / "cameras.bin", "rb").read()
    assert b == struct.pack("<QiiQQ4d", 1, 4, 2, 640, 480, 1.0, 2.0, 3.0, 4.0)
    assert open(tmp_path / "points3D.bin", "rb").read() == struct.pack("<Q", 0)


def test_binary_round_trip(tmp_path):
    rec = random_rec()
    colmap.write_bin_dir(rec, str(tmp_path))
    back = colmap.read_bin_dir(str(tmp_path))
    assert_rec_equal(rec, back)  # binary reader keeps file order (no sort)
    assert_rec_equal(rec, colmap.read_dir_any(str(tmp_path)))
    with open(tmp_path / "cameras.bin", "r+b") as f:
        f.seek(12)
        f.write(struct.pack("<i", 42))  # unknown model id
    with pytest.raises(RcmvsError):
        colmap.read_bin_dir(str(tmp_path))


def test_text_round_trip_sorts(tmp_path):
    rec = random_rec(1)
    colmap.write_txt_dir(rec, str(tmp_path))
    back = colmap.read_txt_dir(str(tmp_path))
    rec.sort_all()
    assert_rec_equal(rec, back)


def test_text_reader_quirks(tmp_path):
    (tmp_path / "cameras.txt").write_text("# comment\n2 simple_pinhole 100 50 60.5 50 25\n9 bad\n")
    (tmp_path / "images.txt").write_text("# c\n5 1 0 0 0 0.5 -1 2 2 my image.png\n\n"
                                         "3 1 0 0 0 0 0 0 2 x.png\n1.5 2.5 -1 4 5\n")
    (tmp_path / "points3D.txt").write_text("# c\n8 1 2 3 300 2 3 0.5 5 7 3\n1 0 0 0 1 2 3 0.1\n")
    rec = colmap.read_txt_dir(str(tmp_path))
    assert [(c.camera_id, c.model_id, c.params) for c in rec.cameras] == [(2, 0, [60.5, 50.0, 25.0])]
    assert [i.image_id for i in rec.images] == [3, 5] and rec.images[1].name == "my image.png"
    assert rec.images[0].xys.tolist() == [[1.5, 2.5]] and rec.images[0].point3d_ids.tolist() == [-1]
    assert rec.images[1].xys.shape == (0, 2)
    assert [p.point3d_id for p in rec.points3d] == [1, 8]
    assert rec.points3d[1].rgb == [300 & 0xFF, 2, 3] and rec.points3d[1].track == [(5, 7)]
    (tmp_path / "cameras.txt").write_text("1 NO_SUCH 10 10 1 2 3\n")
    with pytest.raises(RcmvsError):
        colmap.read_txt_dir(str(tmp_path))


def test_rust_float_display():
    cases = {1.0: "1", 0.1: "0.1", 1e-7: "0.0000001", 1e21: "1000000000000000000000", -0.0: "-0",
             123.456: "123.456", -2.5e-3: "-0.0025", float("nan"): "NaN", float("inf"): "inf"}
    for x, s in cases.items():
        assert colmap._rust_f64(x) == s, (x, colmap._rust_f64(x))


def test_quat_to_rot():
    assert np.array_equal(colmap.quat_to_rot([1, 0, 0, 0]), np.eye(3))
    c = np.cos(np.pi / 4)
    R = colmap.quat_to_rot([c, 0, 0, c])  # 90 degrees about z
    assert np.allclose(R, [[0, -1, 0], [1, 0, 0], [0, 0, 1]], atol=1e-15)
    R2 = colmap.quat_to_rot([2.0, 0, 0, 2.0])  # not unit: normalised first
    assert np.allclose(R2, R, atol=1e-15)
    rng = np.random.default_rng(3)
    q = rng.normal(size=4)
    R3 = colmap.quat_to_rot(q)
    assert np.allclose(R3 @ R3.T, np.eye(3), atol=1e-12) and abs(np.linalg.det(R3) - 1) < 1e-12


def test_cam_from_rec_models():
    p = [10.0, 20.0, 30.0, 40.0, 0.1, 0.2, 0.3, 0.4]
    sx, sy = 0.5, 0.25
    s = 0.5 * (sx + sy)
    expect = {colmap.SIMPLE_PINHOLE: (10, 20, 30, 0), colmap.SIMPLE_RADIAL: (10, 20, 30, 40),
              colmap.RADIAL: (10, 30, 40, 0), colmap.PINHOLE: (15, 30, 40, 0), colmap.OPENCV: (15, 30, 40, 0),
              6: (10, 30, 40, 0)}
    for mid, (f, cx, cy, k) in expect.items():
        c = colmap.cam_from_rec(colmap.Camera(1, mid, 100, 100, p[:colmap._BY_ID[mid][2]]), sx, sy)
        assert (c.f, c.cx, c.cy, c.k) == (f * s, cx * sx, cy * sy, k), mid


def test_working_size():
    assert colmap.working_size(1920, 1080, 4096) == (1920, 1080)
    assert colmap.working_size(1920, 1080, 960) == (960, 540)
    assert colmap.working_size(1000, 10, 100) == (100, 16)
    # f64::round goes half away from zero: 997 * 0.5 = 498.5 -> 499
    assert colmap.working_size(1000, 997, 500) == (500, 499)
    assert colmap.working_size(3, 3, 0) == (16, 16)


def test_working_size_c_abi_agrees():
    """rcmvs_working_size (host C, no GPU) against the Python restatement."""
    rng = np.random.default_rng(3)
    cases = [(1000, 997, 500), (4000, 3000, 900), (17, 9, 1), (8388608, 3, 4096)]
    cases += [tuple(int(v) for v in rng.integers(1, 9000, 2)) + (int(rng.integers(0, 5000)),) for _ in range(300)]
    for w, h, m in cases:
        assert mvs.working_size(w, h, m) == colmap.working_size(w, h, m), (w, h, m)
    with pytest.raises(mvs.RcmvsError):
        mvs.working_size(0, 5, 100)


def _png(img, filt):
    """Test encoder: 8-bit PNG with one filter type on every row."""
    h, w, c = img.shape
    ctype = {1: 0, 2: 4, 3: 2, 4: 6}[c]
    x = img.reshape(h, w * c).astype(np.int32)
    rows = []
    for y in range(h):
        cur, prev = x[y], (x[y - 1] if y else np.zeros(w * c, np.int32))
        a = np.concatenate([np.zeros(c, np.int32), cur[:-c]])
        cc = np.concatenate([np.zeros(c, np.int32), prev[:-c]])
        if filt == 0:
            f = cur
        elif filt == 1:
            f = cur - a
        elif filt == 2:
            f = cur - prev
        elif filt == 3:
            f = cur - ((a + prev) >> 1)
        else:
            p = a + prev - cc
            pa, pb, pc = np.abs(p - a), np.abs(p - prev), np.abs(p - cc)
            f = cur - np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, prev, cc))
        rows.append(bytes([filt]) + (f & 0xFF).astype(np.uint8).tobytes())

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(b"".join(rows))) + chunk(b"IEND", b""))


def test_png_decoder_all_filters(tmp_path):
    rng = np.random.default_rng(4)
    for c in (1, 2, 3, 4):
        img = rng.integers(0, 256, (5, 7, c), dtype=np.uint8)
        for filt in range(5):
            p = tmp_path / f"x{c}{filt}.png"
            p.write_bytes(_png(img, filt))
            assert np.array_equal(colmap.read_png(str(p)), img), (c, filt)
    g = rng.integers(0, 256, (9, 4), dtype=np.uint8)
    mvs.write_png_gray(str(tmp_path / "g.png"), g)
    assert np.array_equal(colmap.read_png(str(tmp_path / "g.png"))[:, :, 0], g)
    (tmp_path / "j.jpg").write_bytes(b"\xff\xd8\xff\xe0")
    with pytest.raises(RcmvsError):
        colmap.read_png(str(tmp_path / "j.jpg"))


def test_png_decoders_agree_on_every_filter(tmp_path):
    """read_image decodes PNG with Pillow when it is installed; the pixels
    must be read_png's for every filter type and channel count."""
    pytest.importorskip("PIL")
    rng = np.random.default_rng(5)
    for c in (1, 2, 3, 4):
        img = rng.integers(0, 256, (23, 31, c), dtype=np.uint8)
        for filt in range(5):
            p = tmp_path / f"y{c}{filt}.png"
            p.write_bytes(_png(img, filt))
            a = colmap._png_with_pillow(str(p))
            assert a is not None and np.array_equal(a, colmap.read_png(str(p))), (c, filt)
            assert np.array_equal(colmap.read_image(str(p)), img)


def test_gray_rgb_conversion():
    rgb = np.array([[[255, 255, 255], [10, 20, 30], [0, 0, 255]]], np.uint8)
    g, out = colmap.gray_rgb(rgb)
    assert g.tolist() == [[255, (2126 * 10 + 7152 * 20 + 722 * 30) // 10000, 722 * 255 // 10000]]
    assert np.array_equal(out, rgb)
    grey = np.arange(256, dtype=np.uint8).reshape(16, 16, 1)
    g, out = colmap.gray_rgb(grey)
    assert np.array_equal(g, grey[:, :, 0]) and np.array_equal(out[:, :, 1], grey[:, :, 0])
    grey3 = np.repeat(grey, 3, axis=2)
    assert np.array_equal(colmap.gray_rgb(grey3)[0], grey[:, :, 0])  # luma of grey is the identity


def write_scene_model(sc, d, img_dir):
    """A COLMAP binary model + grey PNGs of a synthetic scene."""
    os.makedirs(img_dir, exist_ok=True)
    cams, imgs = [], []
    for i, v in enumerate(sc.views):
        cams.append(colmap.Camera(i + 1, colmap.SIMPLE_RADIAL, v.w, v.h, [v.cam.f, v.cam.cx, v.cam.cy, v.cam.k]))
        imgs.append(colmap.Image(100 + i, rot_to_quat(v.R), list(v.t), i + 1, v.name))
        mvs.write_png_gray(os.path.join(img_dir, v.name), v.gray)
    off, tv = sc.sparse.track_offsets, sc.sparse.track_views
    pts = [colmap.Point3D(k, list(sc.sparse.xyz[k]), [0, 0, 0], 0.0,
                          [(100 + int(tv[j]), 0) for j in range(int(off[k]), int(off[k + 1]))])
           for k in range(len(sc.sparse.xyz))]
    colmap.write_bin_dir(colmap.Reconstruction(cams, imgs, pts), d)


def _tiny():
    return scene.corner_room(seed=2, n_views=4, w=96, h=64, f=110.0, arc_deg=40.0, n_patches=20, per_view_sparse=60)


def test_load_views_from_written_model(tmp_path):
    sc = _tiny()
    write_scene_model(sc, str(tmp_path / "sparse"), str(tmp_path / "images"))
    rec = colmap.read_dir_any(str(tmp_path / "sparse"))
    views, sparse = colmap.load_views(rec, str(tmp_path / "images"), MvsOptions(max_dim=4096))
    assert len(views) == len(sc.views)
    for a, b in zip(views, sc.views):
        assert a.name == b.name and (a.w, a.h) == (b.w, b.h) and np.array_equal(a.gray, b.gray)
        assert (a.cam.f, a.cam.cx, a.cam.cy, a.cam.k) == (b.cam.f, b.cam.cx, b.cam.cy, b.cam.k)
        assert np.allclose(a.R, b.R, atol=1e-12) and np.array_equal(a.t, np.asarray(b.t, np.float64))
    assert np.array_equal(sparse.xyz, sc.sparse.xyz)
    assert np.array_equal(sparse.track_offsets, sc.sparse.track_offsets)
    assert np.array_equal(sparse.track_views, sc.sparse.track_views)
    rec.images[0].camera_id = 99
    with pytest.raises(RcmvsError, match="missing camera"):
        colmap.load_views(rec, str(tmp_path / "images"), MvsOptions(max_dim=4096))


@pytest.mark.gpu
def test_run_mvs_colmap_end_to_end(tmp_path):
    sc = _tiny()
    write_scene_model(sc, str(tmp_path / "sparse"), str(tmp_path / "images"))
    opts = MvsOptions(max_dim=4096, num_sources=2, sweeps=1, num_hyp=16, min_consistent=1, save_depth_vis=True)
    ctx = mvs.Context(0)
    st, xyz, rgb = colmap.run_mvs_colmap(str(tmp_path / "sparse"), str(tmp_path / "images"), str(tmp_path / "out"),
                                         opts, ctx=ctx)
    views, sparse = colmap.load_views(colmap.read_dir_any(str(tmp_path / "sparse")), str(tmp_path / "images"), opts)
    _, xyz2, rgb2 = mvs.run_mvs(views, sparse, opts, ctx=ctx)
    ctx.close()
    assert len(xyz) > 0 and np.array_equal(xyz, xyz2) and np.array_equal(rgb, rgb2)
    for f in ("dense.ply", "mvs_stats.json", "dense_web.json"):
        assert (tmp_path / "out" / "dense" / f).exists()
    assert len(os.listdir(tmp_path / "out" / "dense" / "depth_vis")) > 0


@pytest.mark.gpu
def test_load_views_resizes_above_max_dim(tmp_path):
    """Cameras larger than max_dim: views come out at the working size, with
    the oracle's resized images and scaled cameras, and the whole run works."""
    from oracle import oracle
    sc = _tiny()
    write_scene_model(sc, str(tmp_path / "sparse"), str(tmp_path / "images"))
    rec = colmap.read_dir_any(str(tmp_path / "sparse"))
    ctx = mvs.Context(0)
    opts = MvsOptions(max_dim=70, num_sources=2, sweeps=1, num_hyp=16, min_consistent=1)
    views, _ = colmap.load_views(rec, str(tmp_path / "images"), opts, ctx=ctx)
    for a, b in zip(views, sc.views):
        mw, mh = colmap.working_size(b.w, b.h, 70)
        assert (a.w, a.h) == (mw, mh) == (70, 47)
        g, rgb = oracle.resize_view(b.gray, mw, mh)
        assert np.array_equal(a.gray, g) and np.array_equal(a.rgb, rgb)
        want = colmap.cam_from_rec(colmap.Camera(1, colmap.SIMPLE_RADIAL, b.w, b.h,
                                                 [b.cam.f, b.cam.cx, b.cam.cy, b.cam.k]), mw / b.w, mh / b.h)
        assert (a.cam.f, a.cam.cx, a.cam.cy, a.cam.k) == (want.f, want.cx, want.cy, want.k)
    st, _, _ = colmap.run_mvs_colmap(str(tmp_path / "sparse"), str(tmp_path / "images"), str(tmp_path / "out"),
                                       opts, ctx=ctx)
    ctx.close()
    assert st.views == len(sc.views) and st.views_with_depth > 0


def test_read_image_formats(tmp_path):
    """PNG through the in-repo decoder, JPEG and BMP through Pillow; modes
    without a direct counterpart come back as RGB."""
    from PIL import Image
    rng = np.random.default_rng(8)
    rgb = rng.integers(0, 256, (21, 34, 3), dtype=np.uint8)
    grey = rgb[:, :, 0].copy()
    Image.fromarray(rgb).save(tmp_path / "a.png")
    Image.fromarray(rgb).save(tmp_path / "a.bmp")
    Image.fromarray(rgb).save(tmp_path / "a.jpg", quality=95)
    Image.fromarray(grey).save(tmp_path / "g.jpg", quality=95)
    Image.fromarray(rgb).convert("P").save(tmp_path / "p.bmp")
    assert np.array_equal(colmap.read_image(str(tmp_path / "a.png")), rgb)
    assert np.array_equal(colmap.read_image(str(tmp_path / "a.bmp")), rgb)
    j = colmap.read_image(str(tmp_path / "a.jpg"))
    assert j.shape == rgb.shape and np.array_equal(j, np.asarray(Image.open(tmp_path / "a.jpg")))
    g = colmap.read_image(str(tmp_path / "g.jpg"))
    assert g.shape == (21, 34, 1)
    p = colmap.read_image(str(tmp_path / "p.bmp"))
    assert p.shape == (21, 34, 3)
    (tmp_path / "bad.jpg").write_bytes(b"not an image")
    with pytest.raises(RcmvsError):
        colmap.read_image(str(tmp_path / "bad.jpg"))


def test_load_views_from_jpeg_model(tmp_path):
    from PIL import Image
    sc = _tiny()
    write_scene_model(sc, str(tmp_path / "sparse"), str(tmp_path / "images"))
    rec = colmap.read_dir_any(str(tmp_path / "sparse"))
    for im in rec.images:  # the same model with JPEG files
        v = sc.views[im.image_id - 100]
        name = os.path.splitext(im.name)[0] + ".jpg"
        Image.fromarray(np.ascontiguousarray(v.rgb)).save(tmp_path / "images" / name, quality=98)
        im.name = name
    views, _ = colmap.load_views(rec, str(tmp_path / "images"), MvsOptions(max_dim=4096))
    for a, b in zip(views, sc.views):
        assert (a.w, a.h) == (b.w, b.h)
        assert np.abs(a.rgb.astype(int) - np.asarray(b.rgb, int)).mean() < 4.0  # lossy, but close
