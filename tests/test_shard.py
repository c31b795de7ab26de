"""Single-scene multi-GPU host logic (rustcolmap_b200.shard) with world-size 2
and 3 `gloo` process groups on the CPU: view assignment, the depth-map and
candidate all-gathers, and the sharded pipeline (stereo and fusion) against
the single-process one (with the CPU oracle standing in for the GPU stereo,
fusion candidates and voxel dedup).  The split of fusion itself (candidates
of view subsets, concatenated in view order, then the dedup) is checked
against whole fusion on the oracle here and on the GPU."""
import multiprocessing as mp
import os
import socket
import tempfile

import numpy as np
import pytest

from rustcolmap_b200 import scene, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(fn, world, *args):
    """Runs fn(rank, world, outdir, *args) in `world` spawned processes joined
    by a gloo group on 127.0.0.1; returns the outdir."""
    port = _free_port()
    out = tempfile.mkdtemp()
    ctx = mp.get_context("spawn")
    ps = [ctx.Process(target=_entry, args=(fn, r, world, port, out) + args) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(240)
    for p in ps:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in ps), [p.exitcode for p in ps]
    return out


def _entry(fn, rank, world, port, out, *args):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        fn(rank, world, out, *args)
    finally:
        dist.destroy_process_group()


def test_assign_views_partitions_and_balances():
    rng = np.random.default_rng(0)
    costs = [int(c) for c in rng.integers(1, 100, 37)]
    for world in (1, 2, 3, 8, 50):
        parts = shard.assign_views(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        assert parts == shard.assign_views(costs, world)  # deterministic
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert shard.assign_views([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        shard.assign_views([1], 0)


SHAPES = {0: (3, 5), 1: (7, 2), 2: (1, 1), 4: (6, 6), 5: (2, 9)}


def _map(v):
    return (np.arange(np.prod(SHAPES[v]), dtype=np.float32) * (v + 1) + 0.5).reshape(SHAPES[v])


def _gather_rank(rank, world, out, owners):
    local = {v: _map(v) for v, o in owners.items() if o == rank}
    got = shard.all_gather_maps(local, SHAPES, owners)
    np.savez(os.path.join(out, f"r{rank}.npz"), **{str(k): v for k, v in got.items()})


@pytest.mark.parametrize("world,owners", [
    (2, {0: 0, 1: 1, 2: 1, 4: 0, 5: 1}),
    (3, {0: 2, 1: 2, 2: 0, 4: 2, 5: 0}),  # rank 1 owns nothing
])
def test_all_gather_maps_gloo(world, owners):
    out = _run_ranks(_gather_rank, world, owners)
    for r in range(world):
        got = dict(np.load(os.path.join(out, f"r{r}.npz")))
        assert sorted(got) == sorted(str(v) for v in SHAPES)
        for v in SHAPES:
            assert np.array_equal(got[str(v)], _map(v))


def _tiny():
    from rustcolmap_b200 import MvsOptions
    sc = scene.corner_room(seed=2, n_views=5, w=96, h=64, f=110.0, arc_deg=40.0, n_patches=20, per_view_sparse=60)
    opts = MvsOptions(max_dim=4096, num_sources=2, sweeps=1, num_hyp=8, min_consistent=1)
    return sc, opts


def _csr(order):
    return np.cumsum([0] + [len(f) for f in order]), [x for f in order for x in f]


def _oracle_backends(sc, opts):
    from oracle import oracle

    def stereo(jobs):
        return {r: oracle.estimate_depth(sc.views, r, s, a, b, opts, nthreads=1, normals=False)[0]
                for r, s, a, b in jobs}

    def fuse(depth, order):
        off, flat = _csr(order)
        xyz, rgb, _ = oracle.fuse_depth_maps(sc.views, depth, off, flat, sc.sparse.xyz, opts, nthreads=1)
        return xyz, rgb

    def candidates(depth, order, refs):
        off, flat = _csr(order)
        return oracle.fuse_candidates(sc.views, depth, off, flat, refs, opts, nthreads=1)

    def reduce(xyz, rgb):
        return oracle.fuse_reduce(xyz, rgb, sc.sparse.xyz, opts)
    return stereo, fuse, candidates, reduce


def _reference_run(sc, opts):
    from rustcolmap_b200 import mvs
    stereo, fuse, _, _ = _oracle_backends(sc, opts)
    srcs, zr, fus = mvs.plan(sc.sparse, sc.views, opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(sc.views)) if srcs[i]]
    maps = stereo(jobs)
    depth = [maps.get(i) for i in range(len(sc.views))]
    xyz, rgb = fuse(depth, fus)
    return depth, fus, xyz, rgb


def test_oracle_fusion_split_equals_whole():
    """Candidates of disjoint view subsets, concatenated in view order, then
    the dedup: the cloud of whole fusion, bit for bit."""
    sc, opts = _tiny()
    depth, fus, ref_xyz, ref_rgb = _reference_run(sc, opts)
    _, _, candidates, reduce = _oracle_backends(sc, opts)
    with_map = [i for i, d in enumerate(depth) if d is not None]
    ax, ac, pv = candidates(depth, fus, with_map)
    assert len(ax) > 0 and int(pv.sum()) == len(ax)
    assert all(pv[i] == 0 for i, d in enumerate(depth) if d is None)
    xyz, rgb = reduce(ax, ac)
    assert np.array_equal(xyz, ref_xyz) and np.array_equal(rgb, ref_rgb)
    # subsets: every other view, and the rest
    a, b = with_map[::2], with_map[1::2]
    xa, ca, pa = candidates(depth, fus, a)
    xb, cb, pb = candidates(depth, fus, b)
    assert np.array_equal(pa + pb, pv)
    pieces_x, pieces_c, ia, ib = [], [], 0, 0
    for v in range(len(depth)):
        ka, kb = int(pa[v]), int(pb[v])
        pieces_x += [xa[ia:ia + ka], xb[ib:ib + kb]]
        pieces_c += [ca[ia:ia + ka], cb[ib:ib + kb]]
        ia, ib = ia + ka, ib + kb
    mx, mc = np.concatenate(pieces_x), np.concatenate(pieces_c)
    assert np.array_equal(mx, ax) and np.array_equal(mc, ac)
    ex, ec = reduce(np.zeros((0, 3)), np.zeros((0, 3), np.uint8))
    assert ex.shape == (0, 3) and ec.shape == (0, 3)


def _cand_rank(rank, world, out, n_views, counts):
    rng = np.random.default_rng(100 + rank)
    pv = np.array(counts[rank], np.int64)
    n = int(pv.sum())
    xyz = rng.normal(size=(n, 3))
    rgb = rng.integers(0, 256, (n, 3), dtype=np.uint8)
    np.savez(os.path.join(out, f"in{rank}.npz"), xyz=xyz, rgb=rgb)
    gx, gc = shard.all_gather_candidates(xyz, rgb, pv)
    np.savez(os.path.join(out, f"r{rank}.npz"), xyz=gx, rgb=gc)


@pytest.mark.parametrize("world,counts", [
    (2, [[3, 0, 2, 0, 0], [0, 4, 0, 0, 1]]),
    (3, [[0, 0, 0, 0], [5, 0, 0, 2], [0, 0, 0, 0]]),  # ranks with no candidates
])
def test_all_gather_candidates_gloo(world, counts):
    n_views = len(counts[0])
    out = _run_ranks(_cand_rank, world, n_views, counts)
    ins = [dict(np.load(os.path.join(out, f"in{r}.npz"))) for r in range(world)]
    want_x, want_c, cur = [], [], [0] * world
    for v in range(n_views):
        for r in range(world):
            k = counts[r][v]
            want_x.append(ins[r]["xyz"][cur[r]:cur[r] + k])
            want_c.append(ins[r]["rgb"][cur[r]:cur[r] + k])
            cur[r] += k
    wx, wc = np.concatenate(want_x), np.concatenate(want_c)
    for r in range(world):
        got = dict(np.load(os.path.join(out, f"r{r}.npz")))
        assert np.array_equal(got["xyz"], wx) and np.array_equal(got["rgb"], wc)


def _pipeline_rank(rank, world, out):
    sc, opts = _tiny()
    stereo, _, candidates, reduce = _oracle_backends(sc, opts)
    xyz, rgb, depth = shard.run_mvs_sharded(sc.views, sc.sparse, opts, stereo=stereo, candidates=candidates,
                                            reduce=reduce)
    np.savez(os.path.join(out, f"r{rank}.npz"), xyz=xyz, rgb=rgb,
             **{f"d{i}": d for i, d in enumerate(depth) if d is not None})


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_pipeline_equals_single_process(world):
    """Ranks, each running the oracle's stereo and consistency check on its
    share of the views, end with the same depth maps and fused cloud as one
    process running all views."""
    sc, opts = _tiny()
    ref_depth, _, ref_xyz, ref_rgb = _reference_run(sc, opts)
    assert len(ref_xyz) > 0
    out = _run_ranks(_pipeline_rank, world)
    for r in range(world):
        got = dict(np.load(os.path.join(out, f"r{r}.npz")))
        assert np.array_equal(got["xyz"], ref_xyz) and np.array_equal(got["rgb"], ref_rgb)
        for i, d in enumerate(ref_depth):
            if d is not None:
                assert np.array_equal(got[f"d{i}"].view(np.uint32), d.view(np.uint32))


@pytest.mark.gpu
def test_sharded_run_on_one_gpu_equals_run_mvs():
    """World size 1 on the GPU: the sharded driver gives run_mvs's cloud."""
    import torch.distributed as dist
    from rustcolmap_b200 import mvs
    sc, opts = _tiny()
    ctx = mvs.Context(0)
    _, xa, ca = mvs.run_mvs(sc.views, sc.sparse, opts, ctx=ctx)
    port = _free_port()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        xb, cb, _ = shard.run_mvs_sharded(sc.views, sc.sparse, opts, ctx=ctx)
    finally:
        dist.destroy_process_group()
    ctx.close()
    assert np.array_equal(xa, xb) and np.array_equal(ca, cb)


# ------------------------------------------------------------ SfM front end
def _sfm_images():
    sc = scene.corner_room(seed=6, n_views=5, w=120, h=90, f=140.0, arc_deg=30.0, n_patches=30, per_view_sparse=10)
    return [np.ascontiguousarray(v.rgb) for v in sc.views]


def _sfm_backends():
    from oracle import oracle
    from rustcolmap_b200 import colmap, sift

    def extract(im, name):
        g, rgb = colmap.gray_rgb(im)
        pts, desc, col, nraw = oracle.extract_sift(g, rgb)
        return sift.SiftFrame(name, im.shape[1], im.shape[0], pts, desc, col, nraw)

    def match(descs, prs):
        return [oracle.match_pair(descs[i], descs[j], 0.75) for i, j in prs]
    return extract, match


def _sfm_rank(rank, world, out, sequential):
    extract, match = _sfm_backends()
    frames, pairs, matches = shard.extract_and_match_sharded(_sfm_images(), sequential=sequential,
                                                             extract=extract, match=match)
    np.savez(os.path.join(out, f"r{rank}.npz"), pairs=np.array(pairs),
             **{f"p{i}": f.pts for i, f in enumerate(frames)}, **{f"d{i}": f.desc for i, f in enumerate(frames)},
             **{f"c{i}": f.colors for i, f in enumerate(frames)},
             **{f"a{p}": a for p, (a, _) in enumerate(matches)}, **{f"b{p}": b for p, (_, b) in enumerate(matches)})


@pytest.mark.parametrize("world,sequential", [(2, False), (3, True)])
def test_sfm_front_end_sharded_equals_single_process(world, sequential):
    from rustcolmap_b200 import sift
    extract, match = _sfm_backends()
    imgs = _sfm_images()
    frames = [extract(im, "") for im in imgs]
    pairs = sift.job_pairs(len(imgs), sequential)
    ref = match([f.desc for f in frames], pairs)
    assert sum(len(a) for a, _ in ref) > 0
    out = _run_ranks(_sfm_rank, world, sequential)
    for r in range(world):
        got = dict(np.load(os.path.join(out, f"r{r}.npz")))
        assert [tuple(p) for p in got["pairs"]] == pairs
        for i, f in enumerate(frames):
            assert np.array_equal(got[f"p{i}"], f.pts) and np.array_equal(got[f"c{i}"], f.colors)
            assert np.array_equal(got[f"d{i}"].view(np.uint32), f.desc.view(np.uint32))
        for p, (a, b) in enumerate(ref):
            assert np.array_equal(got[f"a{p}"], a) and np.array_equal(got[f"b{p}"], b)


# ------------------------------------------------- device data plane
class _OracleOps:
    """shard.SceneOps' interface with the CPU oracle behind it and CPU
    tensors standing in for device memory (the gloo tests)."""

    def __init__(self, sc, opts):
        from oracle import oracle
        self.o, self.sc, self.opts, self.maps = oracle, sc, opts, {}

    def stereo(self, jobs):
        for r, s, a, b in jobs:
            self.maps[r] = self.o.estimate_depth(self.sc.views, r, s, a, b, self.opts, nthreads=1, normals=False)[0]

    def depth_into(self, v, t):
        import torch
        t.copy_(torch.from_numpy(self.maps[v].ravel()))

    def set_depth(self, v, t):
        v_ = self.sc.views[v]
        self.maps[v] = t.numpy().reshape(v_.h, v_.w).copy()

    def candidates(self, order, refs):
        off, flat = _csr(order)
        depth = [self.maps.get(i) for i in range(len(self.sc.views))]
        self.cx, self.cc, pv = self.o.fuse_candidates(self.sc.views, depth, off, flat, refs, self.opts, nthreads=1)
        return len(self.cx), pv

    def candidates_into(self, x, c):
        import torch
        n = len(self.cx)
        x[:n] = torch.from_numpy(self.cx)
        c[:n] = torch.from_numpy(self.cc)

    def reduce(self, x, c, n, sparse_xyz):
        return self.o.fuse_reduce(x.numpy(), c.numpy(), sparse_xyz, self.opts)

    def depth_host(self, v):
        return self.maps[v]

    def sync(self):
        pass


def _device_plane_rank(rank, world, out):
    from oracle import oracle
    sc, opts = _tiny()
    xyz, rgb, depth = shard.run_mvs_sharded_device(sc.views, sc.sparse, opts, ops=_OracleOps(sc, opts),
                                                   planner=oracle.plan, device="cpu", return_depth=True)
    np.savez(os.path.join(out, f"r{rank}.npz"), xyz=xyz, rgb=rgb,
             **{f"d{i}": d for i, d in enumerate(depth) if d is not None})


@pytest.mark.parametrize("world", [2, 3])
def test_device_data_plane_equals_single_process(world):
    """The device data plane's steps (depth maps into one send tensor, one
    all_gather, maps into every rank's scene; candidates counted, gathered
    as f64 positions and u8 colours, cut and concatenated in view order,
    deduped), run with the oracle behind the scene operations and CPU
    tensors: every rank ends with the single-process maps and cloud."""
    sc, opts = _tiny()
    ref_depth, _, ref_xyz, ref_rgb = _reference_run(sc, opts)
    out = _run_ranks(_device_plane_rank, world)
    for r in range(world):
        got = dict(np.load(os.path.join(out, f"r{r}.npz")))
        assert np.array_equal(got["xyz"], ref_xyz) and np.array_equal(got["rgb"], ref_rgb)
        for i, d in enumerate(ref_depth):
            if d is not None:
                assert np.array_equal(got[f"d{i}"].view(np.uint32), d.view(np.uint32))


@pytest.mark.gpu
def test_device_data_plane_on_one_gpu_equals_run_mvs():
    """World size 1 on the GPU, an NCCL group, the library behind the scene
    operations (depth maps and candidates through device tensors): run_mvs's
    depth maps and cloud."""
    import torch.distributed as dist
    from rustcolmap_b200 import mvs
    sc, opts = _tiny()
    ctx = mvs.Context(0)
    _, xa, ca, da = mvs.run_mvs(sc.views, sc.sparse, opts, ctx=ctx, return_depth=True)
    import datetime

    import torch
    torch.cuda.set_device(0)
    port = _free_port()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        xb, cb, db = shard.run_mvs_sharded_device(sc.views, sc.sparse, opts, ctx=ctx, return_depth=True)
    finally:
        dist.destroy_process_group()
    ctx.close()
    assert np.array_equal(xa, xb) and np.array_equal(ca, cb)
    for a, b in zip(da, db):
        if b is not None:
            assert np.array_equal(a.depth.view(np.uint32), b.view(np.uint32))
