"""Depth-map visualisation (fuse::save_depth_vis, mvs/src/fuse.rs:241-268):
the oracle against hand-derived answers and an independent numpy
restatement, the grey PNG writer, and the GPU image against the oracle."""
import os
import struct
import zlib

import numpy as np
import pytest

from oracle import oracle
from rustcolmap_b200 import mvs


def vis_numpy(depth):
    """Second restatement: numpy f32 scalars, the reference's steps."""
    d = np.asarray(depth, dtype=np.float32)
    ds = np.sort(d[d > 0])
    if len(ds) >= 32:
        lo, hi = ds[int(len(ds) * 0.02)], ds[int(len(ds) * 0.98) - 1]
    else:
        lo, hi = np.float32(0.0), np.float32(1.0)
    rng = max(np.float32(hi - lo), np.float32(1e-9))
    out = np.zeros(d.shape, np.uint8)
    for idx, z in np.ndenumerate(d):
        if z <= 0:
            continue
        t = np.float32((z - lo) / rng)
        t = np.float32(min(max(t, np.float32(0.0)), np.float32(1.0)))
        out[idx] = int(np.float32(np.float32(255.0) * (np.float32(1.0) - t)))
    return out, float(lo), float(hi)


def read_png_gray(path):
    b = open(path, "rb").read()
    assert b[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = None
    while pos < len(b):
        n, = struct.unpack(">I", b[pos:pos + 4])
        typ, data = b[pos + 4:pos + 8], b[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", b[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + data) & 0xFFFFFFFF
        if typ == b"IHDR":
            w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", data)
            assert (depth, ctype, comp, filt, inter) == (8, 0, 0, 0, 0)
        elif typ == b"IDAT":
            idat += data
        elif typ == b"IEND":
            break
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, w + 1)
    assert (raw[:, 0] == 0).all()  # filter type 0 on every row
    return raw[:, 1:].copy()


def maps():
    rng = np.random.default_rng(5)
    a = rng.uniform(1.0, 9.0, (37, 53)).astype(np.float32)
    a[rng.uniform(size=a.shape) < 0.3] = 0.0
    few = np.zeros((8, 9), np.float32)
    few.flat[[3, 10, 40]] = [0.25, 0.75, 3.0]            # < 32 valid: lo 0, hi 1
    ties = np.full((16, 16), 4.0, np.float32)             # range clamps to 1e-9
    ties[0, :5] = 0.0
    ramp = np.arange(1, 101, dtype=np.float32).reshape(10, 10)
    neg = rng.normal(2.0, 2.0, (20, 30)).astype(np.float32)  # negatives are invalid
    empty = np.zeros((5, 7), np.float32)
    return {"random": a, "few": few, "ties": ties, "ramp": ramp, "neg": neg, "empty": empty}


# ------------------------------------------------------------------ CPU
def test_oracle_known_answers():
    m = maps()
    img, lo, hi = oracle.depth_vis(m["ramp"])     # ds = 1..100
    assert (lo, hi) == (3.0, 98.0)                 # ds[2], ds[97]
    assert img[0, 2] == 255 and img[9, 7] == 0 and img[9, 9] == 0 and img[0, 0] == 255
    assert img[4, 9] == int(np.float32(255.0) * (np.float32(1.0) - np.float32(47.0) / np.float32(95.0)))
    img, lo, hi = oracle.depth_vis(m["few"])
    assert (lo, hi) == (0.0, 1.0)
    assert img.flat[3] == 191 and img.flat[10] == 63 and img.flat[40] == 0 and img.sum() == 191 + 63
    img, _, _ = oracle.depth_vis(m["empty"])
    assert not img.any()


def test_oracle_matches_numpy_restatement():
    for name, d in maps().items():
        a = oracle.depth_vis(d)
        b = vis_numpy(d)
        assert np.array_equal(a[0], b[0]), name
        assert a[1:] == b[1:], name


def test_png_writer_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    for h, w in ((1, 1), (7, 13), (64, 3)):
        img = rng.integers(0, 256, (h, w), dtype=np.uint8)
        p = str(tmp_path / f"x{h}_{w}.png")
        mvs.write_png_gray(p, img)
        assert np.array_equal(read_png_gray(p), img)
    with pytest.raises(mvs.RcmvsError):
        mvs.write_png_gray(str(tmp_path / "no_such_dir" / "x.png"), img)


def test_vis_stem():
    assert mvs._vis_stem("images/IMG_001.JPG") == "IMG_001"
    assert mvs._vis_stem("a.b.png") == "a.b"
    assert mvs._vis_stem("") == "view"


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def ctx():
    c = mvs.Context(0)
    yield c
    c.close()


@pytest.mark.gpu
def test_gpu_depth_vis_matches_oracle(ctx):
    ms = maps()
    rng = np.random.default_rng(9)
    big = rng.uniform(2.0, 12.0, (1080, 1920)).astype(np.float32)
    big[rng.uniform(size=big.shape) < 0.6] = 0.0
    ms["big"] = big
    for _ in range(2):  # second call reuses the scratch
        for name, d in ms.items():
            g = mvs.depth_vis(d, ctx)
            o = oracle.depth_vis(d)
            assert np.array_equal(g[0], o[0]), name
            assert g[1:] == o[1:], name


@pytest.mark.gpu
def test_scene_depth_vis_and_run_mvs_pngs(ctx, corner_scene, c1_opts, tmp_path):
    import dataclasses
    v = corner_scene.views
    srcs, zr, _ = mvs.plan(corner_scene.sparse, v, c1_opts)
    ds = mvs.DeviceScene(v, ctx)
    ds.estimate([(2, srcs[2], zr[2, 0], zr[2, 1])], c1_opts)
    img, lo, hi = ds.depth_vis(2)
    o = oracle.depth_vis(ds.depth(2).depth)
    assert np.array_equal(img, o[0]) and (lo, hi) == o[1:]
    with pytest.raises(mvs.RcmvsError):
        ds.depth_vis(3)  # no depth map yet
    ds.close()
    opts = dataclasses.replace(c1_opts, save_depth_vis=True)
    _, _, _, dms = mvs.run_mvs(v, corner_scene.sparse, opts, out_dir=str(tmp_path), ctx=ctx, return_depth=True)
    vis = tmp_path / "dense" / "depth_vis"
    files = sorted(os.listdir(vis))
    assert files == sorted(f"{mvs._vis_stem(x.name)}_depth.png" for i, x in enumerate(v) if srcs[i])
    for i, x in enumerate(v):
        if srcs[i]:
            got = read_png_gray(str(vis / f"{mvs._vis_stem(x.name)}_depth.png"))
            assert np.array_equal(got, oracle.depth_vis(dms[i].depth)[0])
