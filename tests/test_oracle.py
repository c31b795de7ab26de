"""CPU oracle: known answers derived from the reference's semantics, and the
golden vectors of the independent pure-Python restatement
(tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from conftest import golden_views
from oracle import oracle
from rustcolmap_b200 import MvsOptions
from rustcolmap_b200.types import Cam, SparseModel, ViewData

ALL48 = ((1 << 49) - 1) & ~(1 << 24)


def test_census_flat_is_zero():
    assert not oracle.census_map(np.full((9, 11), 77, np.uint8)).any()


def test_census_bright_centre_sets_all_48_bits():
    g = np.zeros((7, 7), np.uint8)
    g[3, 3] = 200
    c = oracle.census_map(g)
    assert int(c[3, 3]) == ALL48
    assert bin(int(c[3, 3])).count("1") == 48


def test_census_strict_less_and_bit_layout():
    # one darker neighbour at (dx, dy) = (+2, -1): bit (dy+3)*7 + (dx+3) = 2*7+5 = 19
    g = np.full((7, 7), 100, np.uint8)
    g[2, 5] = 99
    assert int(oracle.census_map(g)[3, 3]) == 1 << 19
    g[2, 5] = 100  # equal is not darker
    assert int(oracle.census_map(g)[3, 3]) == 0


def test_census_border_clamps():
    # at (0, 0) every dx<0 / dy<0 neighbour clamps onto row/column 0
    g = np.full((5, 5), 50, np.uint8)
    g[0, 0] = 60
    g[0, 1] = 10
    c = int(oracle.census_map(g)[0, 0])
    expect = 0
    for dy in range(-3, 4):
        for dx in range(-3, 4):
            if dx == 0 and dy == 0:
                continue
            xx, yy = min(max(dx, 0), 4), min(max(dy, 0), 4)
            if g[yy, xx] < 60:
                expect |= 1 << ((dy + 3) * 7 + (dx + 3))
    assert c == expect
    # dx = -1..-3 at dy = 0 clamp to (0, 0) itself -> never darker
    for dx in (-3, -2, -1):
        assert not (c >> (3 * 7 + dx + 3)) & 1


def test_census_random_never_sets_bit_24(golden):
    rng = np.random.default_rng(1)
    c = oracle.census_map(rng.integers(0, 256, (31, 29), dtype=np.uint8))
    assert not (c & np.uint64(1 << 24)).any()
    assert (c < np.uint64(1 << 49)).all()


def test_census_matches_python_restatement(golden):
    for i in range(3):
        assert np.array_equal(oracle.census_map(golden[f"gray{i}"]), golden[f"census{i}"])


def test_rng_matches_python_restatement(golden):
    assert oracle.pixel_rng(3, 5, 9) == int(golden["rng_seed_3_5_9"][0])
    u = oracle.rng_stream(3, 5, 9, 4, "u64")
    assert [int(x) for x in u] == [int(x) for x in golden["rng_u64"]]
    import ctypes as C
    s = C.c_uint64(oracle.pixel_rng(3, 5, 9))
    L = oracle.lib()
    for _ in range(4):
        L.orc_next_u64(C.byref(s))
    gs = [L.orc_gauss(C.byref(s)) for _ in range(4)]
    assert np.array_equal(np.array(gs, np.float32), golden["rng_gauss"])


def test_uniform_and_gauss_ranges():
    u = np.array(oracle.rng_stream(7, 1, 11, 5000, "uniform"), np.float32)
    assert (u >= 0).all() and (u < 1).all()
    # (x >> 40) / 2^24 is exact: every value is a multiple of 2^-24
    assert np.array_equal(u * np.float32(1 << 24), np.floor(u * np.float32(1 << 24)))
    g = np.array(oracle.rng_stream(7, 1, 11, 5000, "gauss"), np.float32)
    assert (g >= -1.5).all() and (g < 1.5).all()
    assert abs(float(g.mean())) < 0.05 and 0.4 < float(g.std()) < 0.6


@pytest.mark.parametrize("v,expect", [(float("nan"), 0), (3e9, 2147483647), (-3e9, -2147483648), (-0.5, 0),
                                      (2.99, 2), (-2.99, -2), (float("inf"), 2147483647),
                                      (float("-inf"), -2147483648), (-0.0, 0)])
def test_rust_f32_as_i32(v, expect):
    assert oracle.f32_to_i32(v) == expect


def _exact_pair(w=16, h=12, shift=0.0):
    """Two views with the same camera (f = 256, integer principal point) so
    that pixel -> ray -> pixel is exact; the second is translated by `shift`."""
    rng = np.random.default_rng(3)
    gray = rng.integers(0, 256, (h, w), dtype=np.uint8)
    cam = Cam(256.0, 8.0, 6.0, 0.0)
    R = np.eye(3)
    a = ViewData("a", 0, w, h, cam, R, np.zeros(3), gray, None)
    b = ViewData("b", 1, w, h, cam, R, np.array([shift, 0.0, 0.0]), gray.copy(), None)
    return [a, b]


def test_plane_cost_identity_is_zero():
    views = _exact_pair()
    h, w = 12, 16
    planes = np.zeros((h, w, 4), np.float32)
    planes[..., 2] = 1.0
    planes[..., 3] = 3.0
    cost, hs = oracle.plane_cost_field(views, 0, [1], planes, np.full((h, w), np.inf, np.float32))
    assert (cost == 0).all() and (hs == 0).all()


def test_plane_cost_off_image_is_one_or_aborted():
    views = _exact_pair(shift=1000.0)  # everything projects off the source
    h, w = 12, 16
    planes = np.zeros((h, w, 4), np.float32)
    planes[..., 2] = 1.0
    planes[..., 3] = 3.0
    cost, hs = oracle.plane_cost_field(views, 0, [1], planes, np.full((h, w), np.inf, np.float32))
    assert (cost == 1.0).all() and (hs == 25 * 48).all()
    # a finite hint aborts after the first row: 5/5 = 1 > hint + 0.12
    cost, hs = oracle.plane_cost_field(views, 0, [1], planes, np.full((h, w), 0.5, np.float32))
    assert (cost == np.float32(1e9)).all() and (hs == 5 * 48).all()


def test_plane_cost_grazing_plane_counts_full_mismatch():
    views = _exact_pair()
    h, w = 12, 16
    planes = np.zeros((h, w, 4), np.float32)
    planes[..., 0] = 1.0  # n = (1,0,0): denom = rx, < 0.05 for every ray here
    planes[..., 3] = 3.0
    cost, _ = oracle.plane_cost_field(views, 0, [1], planes, np.full((h, w), np.inf, np.float32))
    assert (cost == 1.0).all()


def test_plane_cost_matches_python_restatement(golden):
    views = golden_views(golden)
    cost, hs = oracle.plane_cost_field(views, 0, [1, 2], golden["planes"], golden["hints"])
    assert np.array_equal(cost.view(np.uint32), golden["plane_cost"].view(np.uint32))
    assert np.array_equal(hs, golden["plane_hsum"])
    assert (cost == np.float32(1e9)).any() and (cost < 1).any()  # both outcomes are covered


def test_estimate_depth_matches_python_restatement(golden):
    views = golden_views(golden)
    nh, sw, thr = golden["params"]
    opts = MvsOptions(max_dim=4096, num_hyp=int(nh), sweeps=int(sw), cost_thr=float(thr))
    zmin, zmax = golden["zrange"]
    for ref in range(3):
        d, c, n, _ = oracle.estimate_depth(views, ref, golden[f"srcs{ref}"], zmin, zmax, opts)
        assert np.array_equal(d.view(np.uint32), golden[f"depth{ref}"].view(np.uint32))
        assert np.array_equal(c.view(np.uint32), golden[f"cost{ref}"].view(np.uint32))
        assert np.array_equal(n.view(np.uint32), golden[f"normal{ref}"].view(np.uint32))


def test_estimate_depth_thread_count_does_not_change_bits(corner_scene, c1_opts):
    v = corner_scene.views
    opts = MvsOptions(max_dim=4096, num_sources=2, sweeps=1, num_hyp=8)
    a = oracle.estimate_depth(v, 2, [1, 3], 3.0, 7.0, opts, nthreads=1)
    b = oracle.estimate_depth(v, 2, [1, 3], 3.0, 7.0, opts, nthreads=7)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_estimate_depth_no_sources():
    views = _exact_pair()
    d, c, n, _ = oracle.estimate_depth(views, 0, [], 1.0, 5.0, MvsOptions(max_dim=4096, num_hyp=4, sweeps=1))
    assert (d == 0).all() and (c == 1.0).all()


def test_fuse_matches_python_restatement(golden):
    views = golden_views(golden)
    depths = [golden[f"depth{i}"] for i in range(3)]
    opts = MvsOptions(min_consistent=1, depth_diff=0.03, voxel_rel=0.0015)
    off = [0, 2, 4, 6]
    order = [1, 2, 0, 2, 1, 0]
    xyz, rgb, ncand = oracle.fuse_depth_maps(views, depths, off, order, golden["sparse_xyz"], opts)
    assert ncand == int(golden["fused_candidates"])
    assert np.array_equal(xyz, golden["fused_xyz"])
    assert np.array_equal(rgb, golden["fused_rgb"])
    assert len(xyz) > 0


PLY_HEADER = ("ply\nformat binary_little_endian 1.0\ncomment rustcolmap dense MVS fusion\n"
              "element vertex {}\nproperty float x\nproperty float y\nproperty float z\n"
              "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n")


def test_ply_layout(tmp_path):
    xyz = np.array([[1.5, -2.25, 3.0], [0.1, 0.2, 0.3]])
    rgb = np.array([[1, 2, 3], [250, 128, 0]], np.uint8)
    p = str(tmp_path / "a.ply")
    oracle.write_ply_binary(p, xyz, rgb)
    b = open(p, "rb").read()
    hdr = PLY_HEADER.format(2).encode()
    assert b.startswith(hdr) and len(b) == len(hdr) + 30
    rec = np.frombuffer(b[len(hdr):], dtype=np.dtype([("p", "<f4", 3), ("c", "u1", 3)]))
    assert np.array_equal(rec["p"], xyz.astype(np.float32)) and np.array_equal(rec["c"], rgb)


def _plan_views(n):
    R = np.eye(3)
    return [ViewData(f"v{i}", i, 8, 8, Cam(8.0, 4.0, 4.0), R, np.array([0.0, 0.0, float(i)]),
                     np.zeros((8, 8), np.uint8)) for i in range(n)]


def _sparse(points):
    xyz = np.array([p for p, _ in points], np.float64)
    off = np.zeros(len(points) + 1, np.uint64)
    tv = []
    for i, (_, t) in enumerate(points):
        off[i + 1] = off[i] + len(t)
        tv += t
    return SparseModel(xyz, off, np.array(tv, np.int32))


def test_plan_sources_threshold_ties_and_fusion_order():
    # view 0 shares 12 points with 1, 12 with 2, 15 with 3, 9 with 4 (< 10)
    pts = []
    for other, cnt in ((1, 12), (2, 12), (3, 15), (4, 9)):
        for k in range(cnt):
            pts.append(((0.1 * k, 0.05 * other, 5.0 + 0.01 * k), [0, other]))
    views = _plan_views(5)
    opts = MvsOptions(num_sources=2)
    srcs, zr, fus = oracle.plan(_sparse(pts), views, opts)
    assert srcs[0] == [3, 1]  # descending count; the 12-12 tie keeps ascending index
    assert srcs[4] == []  # 9 shared points: below the >= 10 threshold
    assert srcs[1] == [0] and srcs[3] == [0]
    # fusion order: co-visible views with a depth map, stereo sources first
    assert fus[0] == [3, 1, 2]
    assert fus[4] == []


def test_plan_depth_range_percentiles_and_fallback():
    pts = [((0.0, 0.0, 1.0 + k), [0, 1]) for k in range(20)]
    views = _plan_views(2)
    srcs, zr, _ = oracle.plan(_sparse(pts), views, MvsOptions())
    z0 = np.array([1.0 + k for k in range(20)])  # view 0: t = 0
    lo, hi = z0[int(round(19 * 0.02))], z0[int(round(19 * 0.98))]
    assert zr[0, 0] == lo * 0.8 and zr[0, 1] == hi * 1.25
    # fewer than 8 points seen by a view: 2/98 percentiles of the global
    # |xyz| list (lib.rs:263-273), x0.8 / x1.25
    pts2 = pts + [((0.0, 0.0, 3.0), [0, 2])]
    views3 = _plan_views(3)
    _, zr3, _ = oracle.plan(_sparse(pts2), views3, MvsOptions())
    g = np.sort(np.array([abs(p[0][2]) for p in pts2]))
    assert zr3[2, 0] == g[int(round((len(g) - 1) * 0.02))] * 0.8
    assert zr3[2, 1] == g[int(round((len(g) - 1) * 0.98))] * 1.25
    # degenerate span (hi <= 1.05 lo): last resort, 1/99 percentiles x0.7 / x1.4
    flat = [((0.0, 0.0, 4.0), [0, 1])] * 12
    _, zr4, _ = oracle.plan(_sparse(flat), _plan_views(2), MvsOptions())
    assert zr4[0, 0] == max(4.0 * 0.7, 1e-3) and zr4[0, 1] == 4.0 * 1.4


def test_plan_rejects_tiny_sparse_model():
    with pytest.raises(RuntimeError):
        oracle.plan(_sparse([((0, 0, 1), [0, 1])] * 7), _plan_views(2), MvsOptions())


def test_oracle_header_says_parity_unpinned():
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for f in ("oracle/mvs_oracle.h", "oracle/mvs_oracle.cpp", "oracle/oracle.py"):
        assert "unpinned" in open(os.path.join(here, f)).read().lower()


def saturating_projection_case():
    """Two views: the ref's one valid pixel sees a point 1000 units to the
    side of the source camera and ~2e-6 in front of its image plane, so the
    source projection saturates `as i32` at INT_MAX (fuse.rs:35-37)."""
    w, h = 8, 6
    cam = Cam(100.0, 4.0, 3.0, 0.0)
    src = ViewData("s", 0, w, h, cam, np.eye(3), np.zeros(3), np.zeros((h, w), np.uint8),
                   np.zeros((h, w, 3), np.uint8))
    ref = ViewData("r", 1, w, h, cam, np.eye(3), np.array([-1000.0, 0.0, 5.0]), np.zeros((h, w), np.uint8),
                   np.full((h, w, 3), 9, np.uint8))
    d_src = np.full((h, w), 3.0, np.float32)
    d_ref = np.zeros((h, w), np.float32)
    d_ref[3, 4] = np.float32(5.000002)
    sparse = np.array([[0, 0, 1], [1, 1, 2], [2, 0, 3], [0, 2, 1]], np.float64)
    return [src, ref], [d_src, d_ref], sparse


def test_fuse_saturated_projection_is_off_image():
    views, dms, sparse = saturating_projection_case()
    opts = MvsOptions(min_consistent=0)
    xyz, rgb, ncand = oracle.fuse_depth_maps(views, [None, dms[1]], [0, 0, 0], [], sparse, opts)
    assert ncand == 1 and len(xyz) == 1  # kept with zero confirmations, no read outside the map
    opts = MvsOptions(min_consistent=1)
    xyz, rgb, ncand = oracle.fuse_depth_maps(views, dms, [0, 0, 1], [0], sparse, opts)
    assert ncand == 0
