"""GPU parity: the librcmvs kernels, called through the C ABI, against the CPU
oracle on the same seeded inputs.  Integer work (census, Hamming sums, RNG)
and the f32 cost/depth/normal maps must be bit-identical; fused points must
be identical as sorted sets."""
import numpy as np
import pytest

from conftest import golden_views
from oracle import oracle
from rustcolmap_b200 import MvsOptions, mvs, scene
from rustcolmap_b200.types import FLAG_LOCKSTEP_PASSES

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def assert_bits_equal(a, b, what=""):
    a, b = bits(a), bits(b)
    if not np.array_equal(a, b):
        bad = np.argwhere(a != b)
        raise AssertionError(f"{what}: {len(bad)} of {a.size} differ, first at {bad[:5].tolist()}")


@pytest.fixture(scope="module")
def ctx():
    c = mvs.Context(0)
    yield c
    c.close()


def test_float_to_int_truncation_semantics(ctx):
    vals = np.array([np.nan, 3e9, -3e9, -0.5, 2.99, -2.99, np.inf, -np.inf, -0.0, 1e-45, 2147483520.0, -0.9999,
                     383.99997, 384.0], np.float32)
    got = mvs.selftest_f2i(vals, ctx)
    assert got.tolist() == [oracle.f32_to_i32(v) for v in vals]


@pytest.mark.parametrize("shape", [(1, 1), (3, 5), (19, 37), (7, 300), (288, 384)])
def test_census_bit_exact(ctx, shape):
    g = np.random.default_rng(shape[0] * 1000 + shape[1]).integers(0, 256, shape, dtype=np.uint8)
    g[: shape[0] // 2, : shape[1] // 3] = 128  # flat area
    assert np.array_equal(mvs.census_map(g, ctx), oracle.census_map(g))


def test_scene_census_bit_exact(ctx, corner_scene):
    ds = mvs.DeviceScene(corner_scene.views, ctx)
    for i in (0, 7):
        assert np.array_equal(ds.census(i), oracle.census_map(corner_scene.views[i].gray))
    ds.close()


def test_plane_cost_field_golden(ctx, golden):
    views = golden_views(golden)
    cost, hs = mvs.plane_cost_field(views, 0, [1, 2], golden["planes"], golden["hints"], ctx)
    assert_bits_equal(cost, golden["plane_cost"], "cost")
    assert np.array_equal(hs, golden["plane_hsum"])


@pytest.mark.parametrize("k", [1, 4])
def test_plane_cost_field_random_planes(ctx, corner_scene, k):
    v = corner_scene.views
    h, w = v[0].h, v[0].w
    rng = np.random.default_rng(k)
    n = rng.normal(size=(h, w, 3)) * [0.5, 0.5, 1.0]
    n[..., 2] = np.abs(n[..., 2])
    n /= np.linalg.norm(n, axis=2, keepdims=True)
    planes = np.concatenate([n, rng.uniform(2.0, 8.0, (h, w, 1))], axis=2).astype(np.float32)
    hints = rng.choice(np.array([np.inf, 0.05, 0.15, 0.3, 0.6], np.float32), size=(h, w))
    srcs = [1, 2, 3, 4][:k]
    c_gpu, h_gpu = mvs.plane_cost_field(v, 0, srcs, planes, hints, ctx)
    c_cpu, h_cpu = oracle.plane_cost_field(v, 0, srcs, planes, hints)
    assert_bits_equal(c_gpu, c_cpu, "plane cost")
    assert np.array_equal(h_gpu, h_cpu)
    assert (c_cpu == np.float32(1e9)).mean() > 0.05 and (c_cpu < 1).mean() > 0.05


def test_estimate_depth_golden(ctx, golden):
    views = golden_views(golden)
    nh, sw, thr = golden["params"]
    opts = MvsOptions(max_dim=4096, num_hyp=int(nh), sweeps=int(sw), cost_thr=float(thr))
    zmin, zmax = golden["zrange"]
    for ref in range(3):
        dm = mvs.estimate_depth(views, ref, golden[f"srcs{ref}"], zmin, zmax, opts, ctx, normals=True)
        assert_bits_equal(dm.depth, golden[f"depth{ref}"], f"depth {ref}")
        assert_bits_equal(dm.cost, golden[f"cost{ref}"], f"cost {ref}")
        assert_bits_equal(dm.normal, golden[f"normal{ref}"], f"normal {ref}")


def _parity_fraction(a, b):
    """Fraction of pixels valid in either map whose inverse depths agree
    within 1e-3 relative (the depth-map tolerance), both invalid counting as
    agreement."""
    va, vb = a > 0, b > 0
    either = va | vb
    both = va & vb
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.abs(1 / a[both] - 1 / b[both]) * b[both]
    ok = int((rel <= 1e-3).sum())
    return ok / max(int(either.sum()), 1)


@pytest.mark.parametrize("ref", [0, 5])
def test_estimate_depth_config1_bit_exact(ctx, corner_scene, c1_opts, ref):
    v = corner_scene.views
    srcs, zr, _ = mvs.plan(corner_scene.sparse, v, c1_opts)
    dm = mvs.estimate_depth(v, ref, srcs[ref], zr[ref, 0], zr[ref, 1], c1_opts, ctx, normals=True)
    d, c, n, _ = oracle.estimate_depth(v, ref, srcs[ref], zr[ref, 0], zr[ref, 1], c1_opts)
    assert _parity_fraction(dm.depth, d) >= 0.99
    assert_bits_equal(dm.depth, d, "depth")
    assert_bits_equal(dm.cost, c, "cost")
    assert_bits_equal(dm.normal, n, "normal")
    m = scene.gt_metrics(dm.depth, corner_scene.gt_depth[ref])
    print(f"\nview {ref}: GT accuracy {m['accuracy']:.3f} completeness {m['completeness']:.3f}")
    assert m["accuracy"] > 0.6


@pytest.mark.parametrize("w,h,srcs,nh,sweeps,tile", [
    (16, 16, [1], 2, 1, (16, 16)),
    (17, 9, [1, 2], 5, 1, (8, 4)),
    (45, 23, [2, 1], 16, 2, (32, 8)),
    (40, 30, [], 8, 1, (16, 16)),
    (61, 7, [1, 2], 8, 1, (32, 1)),
])
def test_estimate_depth_edge_cases(ctx, w, h, srcs, nh, sweeps, tile):
    sc = scene.corner_room(seed=w * h, n_views=3, w=w, h=h, f=1.15 * w, arc_deg=20.0, n_patches=10,
                           per_view_sparse=30)
    opts = MvsOptions(max_dim=4096, num_hyp=nh, sweeps=sweeps, tile_w=tile[0], tile_h=tile[1])
    dm = mvs.estimate_depth(sc.views, 0, srcs, 2.5, 9.0, opts, ctx, normals=True)
    d, c, n, _ = oracle.estimate_depth(sc.views, 0, srcs, 2.5, 9.0, opts)
    assert_bits_equal(dm.depth, d, "depth")
    assert_bits_equal(dm.cost, c, "cost")
    assert_bits_equal(dm.normal, n, "normal")
    if not srcs:
        assert (dm.depth == 0).all() and (dm.cost == 1).all()


@pytest.mark.parametrize("flags", [0, FLAG_LOCKSTEP_PASSES])
def test_max_support_views_bit_exact(ctx, flags):
    """RCMVS_MAX_SOURCES (32) support views: every slot of the streamed
    passes' per-view parameter table is used (and the lockstep kernel's)."""
    sc = scene.orbit_room(seed=33, n_views=33, sizes=((40, 30),), n_boxes=4, per_view_sparse=40, arc_deg=60.0)
    opts = MvsOptions(max_dim=4096, num_hyp=6, sweeps=1, flags=flags)
    srcs = list(range(1, 33))
    dm = mvs.estimate_depth(sc.views, 0, srcs, 1.0, 11.0, opts, ctx, normals=True)
    d, c, n, _ = oracle.estimate_depth(sc.views, 0, srcs, 1.0, 11.0, opts)
    assert_bits_equal(dm.depth, d, "depth")
    assert_bits_equal(dm.cost, c, "cost")
    assert_bits_equal(dm.normal, n, "normal")


def test_tile_shape_does_not_change_bits(ctx, corner_scene):
    v = corner_scene.views
    base = None
    for tw, th in ((16, 16), (8, 8), (32, 4), (64, 2)):
        opts = MvsOptions(max_dim=4096, num_hyp=12, sweeps=1, tile_w=tw, tile_h=th)
        dm = mvs.estimate_depth(v, 3, [2, 4], 3.0, 7.5, opts, ctx)
        if base is None:
            base = dm
        else:
            assert_bits_equal(dm.depth, base.depth)
            assert_bits_equal(dm.cost, base.cost)


def test_batch_equals_single_calls(ctx, corner_scene):
    v = corner_scene.views
    opts = MvsOptions(max_dim=4096, num_hyp=16, sweeps=2)
    jobs = [(1, [0, 2], 3.0, 7.0), (4, [3, 5, 6], 2.8, 7.5), (7, [6], 3.2, 7.2)]
    batch = mvs.estimate_depth_batch(v, jobs, opts, ctx)
    for (ref, srcs, a, b), dm in zip(jobs, batch):
        single = mvs.estimate_depth(v, ref, srcs, a, b, opts, ctx)
        assert_bits_equal(dm.depth, single.depth)
        assert_bits_equal(dm.cost, single.cost)


def test_uneven_batch_bit_exact(ctx):
    """Views of different sizes and support-view counts in one batch."""
    sc = scene.orbit_room(seed=9, n_views=12, sizes=((96, 72), (128, 72), (64, 48)), n_boxes=6,
                          size_choice="random", per_view_sparse=80)
    opts = MvsOptions(max_dim=4096, num_hyp=24, sweeps=2)
    jobs = [(0, [1, 11, 2], 1.0, 11.0), (5, [4, 6], 1.0, 11.0), (9, [8, 10, 7, 11, 0], 1.0, 11.0)]
    batch = mvs.estimate_depth_batch(sc.views, jobs, opts, ctx)
    for (ref, srcs, a, b), dm in zip(jobs, batch):
        d, c, _, _ = oracle.estimate_depth(sc.views, ref, srcs, a, b, opts)
        assert_bits_equal(dm.depth, d, f"depth {ref}")
        assert_bits_equal(dm.cost, c, f"cost {ref}")


@pytest.fixture(scope="module")
def c1_depth(ctx, corner_scene, c1_opts):
    v = corner_scene.views
    srcs, zr, fus = mvs.plan(corner_scene.sparse, v, c1_opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(v))]
    return mvs.estimate_depth_batch(v, jobs, c1_opts, ctx), fus


def _assert_same_cloud(a, b):
    (xa, ca), (xb, cb) = a, b
    assert len(xa) == len(xb)
    assert np.array_equal(xa, xb) and np.array_equal(ca, cb)


@pytest.mark.parametrize("min_cons,ddiff,reproj", [(2, 0.03, 0.0), (3, 0.01, 0.0), (3, 0.01, 1.0), (1, 0.05, 0.0)])
def test_fusion_bit_exact(ctx, corner_scene, c1_depth, min_cons, ddiff, reproj):
    dms, fus = c1_depth
    v = corner_scene.views
    opts = MvsOptions(min_consistent=min_cons, depth_diff=ddiff, reproj_px=reproj)
    off = np.cumsum([0] + [len(f) for f in fus])
    flat = [x for f in fus for x in f]
    g = mvs.fuse_depth_maps(v, [d.depth for d in dms], fus, corner_scene.sparse.xyz, opts, ctx)
    xyz, rgb, ncand = oracle.fuse_depth_maps(v, [d.depth for d in dms], off, flat, corner_scene.sparse.xyz, opts)
    _assert_same_cloud(g, (xyz, rgb))
    assert len(xyz) > 1000


def test_fusion_with_missing_depth_maps(ctx, corner_scene, c1_depth):
    dms, fus = c1_depth
    v = corner_scene.views
    keep = [d.depth if i % 3 else None for i, d in enumerate(dms)]
    fus2 = [[j for j in f if keep[j] is not None] for f in fus]
    opts = MvsOptions(min_consistent=1)
    off = np.cumsum([0] + [len(f) for f in fus2])
    g = mvs.fuse_depth_maps(v, keep, fus2, corner_scene.sparse.xyz, opts, ctx)
    xyz, rgb, _ = oracle.fuse_depth_maps(v, keep, off, [x for f in fus2 for x in f], corner_scene.sparse.xyz, opts)
    _assert_same_cloud(g, (xyz, rgb))


@pytest.mark.parametrize("reproj", [0.0, 1.0])
def test_fusion_split_matches_oracle_and_whole(ctx, corner_scene, c1_depth, reproj):
    """Candidates of view subsets (host and device-resident entry points)
    against the oracle's, and the dedup of all candidates in view order
    against whole fusion."""
    dms, fus = c1_depth
    v = corner_scene.views
    opts = MvsOptions(min_consistent=2, depth_diff=0.02, reproj_px=reproj)
    off = np.cumsum([0] + [len(f) for f in fus])
    flat = [x for f in fus for x in f]
    depth = [d.depth for d in dms]
    whole = mvs.fuse_depth_maps(v, depth, fus, corner_scene.sparse.xyz, opts, ctx)
    for refs in (list(range(len(v))), [0, 3, 5], [7], []):
        gx, gc, gp = mvs.fuse_candidates(v, depth, fus, refs, opts, ctx)
        ox, oc, op = oracle.fuse_candidates(v, depth, off, flat, refs, opts)
        assert np.array_equal(gx, ox) and np.array_equal(gc, oc) and np.array_equal(gp, op), refs
        assert all(gp[i] == 0 for i in range(len(v)) if i not in refs)
    ax, ac, ap = mvs.fuse_candidates(v, depth, fus, list(range(len(v))), opts, ctx)
    _assert_same_cloud(mvs.fuse_reduce(ax, ac, corner_scene.sparse.xyz, opts, ctx), whole)
    _assert_same_cloud(oracle.fuse_reduce(ax, ac, corner_scene.sparse.xyz, opts), whole)
    # two disjoint halves, merged view by view
    a, b = list(range(0, len(v), 2)), list(range(1, len(v), 2))
    xa, ca, pa = mvs.fuse_candidates(v, depth, fus, a, opts, ctx)
    xb, cb, pb = mvs.fuse_candidates(v, depth, fus, b, opts, ctx)
    mx, mc, ia, ib = [], [], 0, 0
    for k in range(len(v)):
        na, nb = int(pa[k]), int(pb[k])
        mx += [xa[ia:ia + na], xb[ib:ib + nb]]
        mc += [ca[ia:ia + na], cb[ib:ib + nb]]
        ia, ib = ia + na, ib + nb
    _assert_same_cloud(mvs.fuse_reduce(np.concatenate(mx), np.concatenate(mc), corner_scene.sparse.xyz, opts, ctx),
                       whole)
    assert len(whole[0]) > 1000
    empty = mvs.fuse_reduce(np.zeros((0, 3)), np.zeros((0, 3), np.uint8), corner_scene.sparse.xyz, opts, ctx)
    assert empty[0].shape == (0, 3)


def test_scene_fuse_candidates_matches_host_entry(ctx, corner_scene, c1_opts):
    """Device-resident candidates after device-resident stereo."""
    v = corner_scene.views
    srcs, zr, fus = mvs.plan(corner_scene.sparse, v, c1_opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(v)) if srcs[i]]
    ds = mvs.DeviceScene(v, ctx)
    ds.estimate(jobs, c1_opts)
    depth = [ds.depth(i).depth if srcs[i] else None for i in range(len(v))]
    refs = [r for r, _, _, _ in jobs][1::2]
    sx, sc_, sp = ds.fuse_candidates(fus, refs, c1_opts)
    hx, hc, hp = mvs.fuse_candidates(v, depth, fus, refs, c1_opts, ctx)
    assert len(sx) > 0 and np.array_equal(sx, hx) and np.array_equal(sc_, hc) and np.array_equal(sp, hp)
    ds.close()


def test_run_mvs_matches_oracle_pipeline(ctx, corner_scene, c1_opts, tmp_path):
    v = corner_scene.views
    stats, xyz, rgb, dms = mvs.run_mvs(v, corner_scene.sparse, c1_opts, out_dir=str(tmp_path), ctx=ctx,
                                       return_depth=True)
    srcs, zr, fus = oracle.plan(corner_scene.sparse, v, c1_opts)
    ref_d = []
    for i in range(len(v)):
        d, _, _, _ = oracle.estimate_depth(v, i, srcs[i], zr[i, 0], zr[i, 1], c1_opts)
        assert_bits_equal(dms[i].depth, d, f"depth {i}")
        ref_d.append(d)
    off = np.cumsum([0] + [len(f) for f in fus])
    oxyz, orgb, ncand = oracle.fuse_depth_maps(v, ref_d, off, [x for f in fus for x in f],
                                               corner_scene.sparse.xyz, c1_opts)
    _assert_same_cloud((xyz, rgb), (oxyz, orgb))
    assert stats.dense_points == len(oxyz) and stats.fusion_candidates == ncand
    body = open(tmp_path / "dense" / "dense.ply", "rb").read()
    assert body.count(b"end_header\n") == 1 and len(body.split(b"end_header\n")[1]) == 15 * len(xyz)
    assert (tmp_path / "dense" / "mvs_stats.json").exists() and (tmp_path / "dense" / "dense_web.json").exists()


def test_device_ply_records_match_host_writer(ctx, corner_scene, c1_depth, c1_opts, tmp_path):
    dms, fus = c1_depth
    ds = mvs.DeviceScene(corner_scene.views, ctx)
    jobs = []
    srcs, zr, _ = mvs.plan(corner_scene.sparse, corner_scene.views, c1_opts)
    for i in range(len(corner_scene.views)):
        jobs.append((i, srcs[i], zr[i, 0], zr[i, 1]))
    ds.estimate(jobs, c1_opts)
    n = ds.fuse(fus, corner_scene.sparse.xyz, c1_opts)
    xyz, rgb, body = ds.points(ply_body=True)
    p = str(tmp_path / "x.ply")
    mvs.write_ply_binary(p, xyz, rgb)
    assert open(p, "rb").read().split(b"end_header\n", 1)[1] == body.tobytes()
    assert n == len(xyz)
    ds.close()


def test_renderer_host_and_device_identical():
    a = scene.orbit_room(seed=4, n_views=3, sizes=((80, 60),), n_boxes=5, n_spheres=3, device=-1)
    b = scene.orbit_room(seed=4, n_views=3, sizes=((80, 60),), n_boxes=5, n_spheres=3, device=0)
    for x, y in zip(a.views, b.views):
        assert np.array_equal(x.gray, y.gray)
    for x, y in zip(a.gt_depth, b.gt_depth):
        assert_bits_equal(x, y)


def test_bad_arguments_raise(ctx, corner_scene):
    v = corner_scene.views
    with pytest.raises(mvs.RcmvsError):
        mvs.estimate_depth(v, 0, [99], 3.0, 7.0, MvsOptions(max_dim=4096), ctx)
    with pytest.raises(mvs.RcmvsError):
        mvs.estimate_depth(v, 0, [1], -1.0, 7.0, MvsOptions(max_dim=4096), ctx)
    with pytest.raises(mvs.RcmvsError):  # views above max_dim are not resized here
        mvs.estimate_depth(v, 0, [1], 3.0, 7.0, MvsOptions(max_dim=100), ctx)
    with pytest.raises(mvs.RcmvsError):
        mvs.estimate_depth(v, 0, list(range(1, 8)) * 5, 3.0, 7.0, MvsOptions(max_dim=4096), ctx)
    with pytest.raises(mvs.RcmvsError):
        mvs.run_mvs(v[:1], corner_scene.sparse, MvsOptions(max_dim=4096), ctx=ctx)


def test_fusion_saturated_projection_matches_oracle(ctx):
    from test_oracle import saturating_projection_case
    views, dms, sparse = saturating_projection_case()
    for mc, order in ((0, [[], []]), (1, [[], [0]])):
        opts = MvsOptions(min_consistent=mc)
        g = mvs.fuse_depth_maps(views, dms if mc else [None, dms[1]], order, sparse, opts, ctx)
        off = np.cumsum([0] + [len(f) for f in order])
        c = oracle.fuse_depth_maps(views, dms if mc else [None, dms[1]], off, [x for f in order for x in f],
                                   sparse, opts)
        _assert_same_cloud(g, c[:2])


@pytest.mark.parametrize("passes,flags", [(1, 0), (3, 0), (5, 0), (5, 16), (7, 256)])
def test_pass_count_extension_matches_oracle(ctx, corner_scene, c1_opts, passes, flags):
    """The passes option (odd counts included, with the perturbation
    annealing over the passes run) gives the oracle's bits, with and without
    the shortcuts."""
    import dataclasses
    v = corner_scene.views
    o = dataclasses.replace(c1_opts, passes=passes, flags=flags)
    srcs, zr, _ = mvs.plan(corner_scene.sparse, v, o)
    for ref in (2, 5):
        d, c, n, _ = oracle.estimate_depth(v, ref, srcs[ref], zr[ref, 0], zr[ref, 1], o)
        g = mvs.estimate_depth(v, ref, srcs[ref], zr[ref, 0], zr[ref, 1], o, ctx, normals=True)
        for x, y in ((g.depth, d), (g.cost, c), (g.normal, n)):
            assert_bits_equal(x, y, f"passes {passes} flags {flags} ref {ref}")


@pytest.mark.parametrize("ref", [1, 6])
def test_row_step_and_one_candidate_kernels_agree(ctx, corner_scene, c1_opts, ref):
    """The default table sweep, the one-candidate-at-a-time kernels
    (RCMVS_FLAG_ONE_CANDIDATE) and the row-step sweep
    (RCMVS_FLAG_ROW_STEP_INIT) give the same bits, and with the shortcuts off
    (RCMVS_FLAG_NO_SKIP_DUPLICATES) the work counters agree with the
    oracle's plane_cost call and row counts."""
    import dataclasses
    import os
    v = corner_scene.views
    srcs, zr, _ = mvs.plan(corner_scene.sparse, v, c1_opts)
    a = mvs.estimate_depth(v, ref, srcs[ref], zr[ref, 0], zr[ref, 1], c1_opts, ctx, normals=True)
    for flags in (1, 128):  # one candidate at a time; the row-step sweep
        o = dataclasses.replace(c1_opts, flags=flags)
        b = mvs.estimate_depth(v, ref, srcs[ref], zr[ref, 0], zr[ref, 1], o, ctx, normals=True)
        for x, y in ((a.depth, b.depth), (a.cost, b.cost), (a.normal, b.normal)):
            assert_bits_equal(x, y, f"flags {flags}")
    os.environ["RCMVS_COUNT"] = "1"
    cctx = mvs.Context(0)
    del os.environ["RCMVS_COUNT"]
    _, _, _, work = oracle.estimate_depth(v, ref, srcs[ref], zr[ref, 0], zr[ref, 1], c1_opts)
    for o in (dataclasses.replace(c1_opts, flags=16), dataclasses.replace(c1_opts, flags=1 | 16),
              dataclasses.replace(c1_opts, flags=128 | 16)):
        ds = mvs.DeviceScene(v, cctx)
        ds.estimate([(ref, srcs[ref], zr[ref, 0], zr[ref, 1])], o)
        assert cctx.last_work() == work
        ds.close()
    cctx.close()


@pytest.mark.parametrize("ref", [2, 5])
def test_duplicate_skip_keeps_bits_and_saves_rows(ctx, corner_scene, c1_opts, ref):
    """Skipping propagated planes that repeat the pixel's own plane bit for
    bit and the planes of neighbours the previous pass left unchanged (the
    default) gives the oracle's bits with fewer window rows than the
    reference's call sequence (RCMVS_FLAG_NO_SKIP_DUPLICATES); the repeat
    skip alone (off with RCMVS_FLAG_NO_REPEAT_SKIP) saves rows too."""
    import dataclasses
    import os
    v = corner_scene.views
    srcs, zr, _ = mvs.plan(corner_scene.sparse, v, c1_opts)
    job = (ref, srcs[ref], zr[ref, 0], zr[ref, 1])
    d, c, n, (evals_ref, rows_ref) = oracle.estimate_depth(v, *job, c1_opts)
    os.environ["RCMVS_COUNT"] = "1"
    cctx = mvs.Context(0)
    del os.environ["RCMVS_COUNT"]
    counts = {}
    for flags in (0, 16, 1, 2 | 4, 128, 128 | 2, 256, 256 | 2 | 4):
        ds = mvs.DeviceScene(v, cctx)
        ds.estimate([job], dataclasses.replace(c1_opts, flags=flags))
        dm = ds.depth(ref, normals=True)
        for got, want in ((dm.depth, d), (dm.cost, c), (dm.normal, n)):
            assert_bits_equal(got, want, f"flags {flags}")
        counts[flags] = cctx.last_work()
        ds.close()
    cctx.close()
    assert counts[16] == (evals_ref, rows_ref)
    assert counts[0] == counts[1] == counts[2 | 4] == counts[128] == counts[128 | 2]
    assert counts[0][1] < 0.9 * rows_ref, (counts[0], rows_ref)
    assert counts[256] == counts[256 | 2 | 4]
    assert counts[0][1] < counts[256][1] < rows_ref, (counts[0], counts[256], rows_ref)
