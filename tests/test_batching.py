"""Batched stereo schedules: persistent (view, tile) work-queue launches,
CUDA-graph replay, per-resolution-class tile shapes (autotuned or loaded)
and cost-ordered jobs.  Each must give the oracle's bits for every view of an
uneven batch (different sizes and support-view counts in one launch)."""
import numpy as np
import pytest

from oracle import oracle
from rustcolmap_b200 import MvsOptions, learned, mvs, scene
from rustcolmap_b200.types import FLAG_AUTOTUNE, FLAG_CUDA_GRAPH, FLAG_LOCKSTEP_PASSES, FLAG_PERSISTENT

pytestmark = pytest.mark.gpu

SIZES = ((96, 72), (128, 72), (64, 48))


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def uneven():
    sc = scene.orbit_room(seed=9, n_views=12, sizes=SIZES, n_boxes=6, size_choice="random", per_view_sparse=80)
    opts = MvsOptions(max_dim=4096, num_hyp=24, sweeps=2)
    # K from 1 to 6, several views per size class
    jobs = [(0, [1, 11, 2], 1.0, 11.0), (5, [4, 6], 1.0, 11.0), (9, [8, 10, 7, 11, 0], 1.0, 11.0),
            (3, [2, 4, 1, 5, 6, 0], 1.2, 10.0), (7, [6], 1.0, 11.0), (10, [9, 11, 8, 0], 0.9, 12.0)]
    ref = {}
    for (r, srcs, a, b) in jobs:
        d, c, n, _ = oracle.estimate_depth(sc.views, r, srcs, a, b, opts)
        ref[r] = (d, c, n)
    return sc, opts, jobs, ref


def _check(ds, jobs, ref, what):
    for (r, _, _, _) in jobs:
        dm = ds.depth(r, normals=True)
        d, c, n = ref[r]
        for got, want, name in ((dm.depth, d, "depth"), (dm.cost, c, "cost"), (dm.normal, n, "normal")):
            gb, wb = bits(got), bits(want)
            assert np.array_equal(gb, wb), f"{what}: view {r} {name}: {(gb != wb).sum()} of {gb.size} differ"


@pytest.mark.parametrize("flags", [0, FLAG_PERSISTENT, FLAG_CUDA_GRAPH, FLAG_PERSISTENT | FLAG_CUDA_GRAPH, 128,
                                   128 | FLAG_PERSISTENT | FLAG_CUDA_GRAPH, FLAG_LOCKSTEP_PASSES,
                                   FLAG_LOCKSTEP_PASSES | FLAG_PERSISTENT | FLAG_CUDA_GRAPH])
def test_schedules_match_oracle(uneven, flags):
    sc, opts, jobs, ref = uneven
    ctx = mvs.Context(0)
    ds = mvs.DeviceScene(sc.views, ctx)
    o = MvsOptions(**{**opts.__dict__, "flags": flags})
    ds.estimate(jobs, o)
    _check(ds, jobs, ref, f"flags {flags}")
    ds.close()
    ctx.close()


def test_graph_replay_and_recapture(uneven):
    sc, opts, jobs, ref = uneven
    ctx = mvs.Context(0)
    ds = mvs.DeviceScene(sc.views, ctx)
    o = MvsOptions(**{**opts.__dict__, "flags": FLAG_CUDA_GRAPH | FLAG_PERSISTENT})
    for _ in range(3):  # capture, then replays of the cached graph
        ds.estimate(jobs, o)
        _check(ds, jobs, ref, "replay")
    # a different job table (depth range, sources, a job less) is recaptured
    jobs2 = [(0, [2, 1], 1.5, 9.0), (9, [8, 10, 7, 11, 0], 1.0, 11.0)]
    ds.estimate(jobs2, o)
    for (r, srcs, a, b) in jobs2:
        d, c, n, _ = oracle.estimate_depth(sc.views, r, srcs, a, b, opts)
        dm = ds.depth(r, normals=True)
        assert np.array_equal(bits(dm.depth), bits(d)) and np.array_equal(bits(dm.cost), bits(c))
    ds.estimate(jobs, o)
    _check(ds, jobs, ref, "after recapture")
    ds.close()
    ctx.close()


@pytest.mark.parametrize("table", [
    # same pixel count, different shapes per class
    {(96, 72): (16, 16), (128, 72): (64, 4), (64, 48): (8, 32)},
    # different pixel counts in one launch: blocks of 256 threads, the 8x8
    # and 32x4 tiles leave threads idle
    {(96, 72): (8, 8), (128, 72): (16, 16), (64, 48): (32, 4)},
    # one warp per tile
    {(96, 72): (8, 4), (128, 72): (4, 8), (64, 48): (16, 2)},
])
@pytest.mark.parametrize("persistent", [False, True])
def test_per_class_tile_shapes_in_one_launch(uneven, table, persistent):
    sc, opts, jobs, ref = uneven
    ctx = mvs.Context(0)
    ctx.set_tune_table([dict(w=w, h=h, tile_w=tw, tile_h=th) for (w, h), (tw, th) in table.items()])
    ds = mvs.DeviceScene(sc.views, ctx)
    o = MvsOptions(**{**opts.__dict__, "flags": FLAG_AUTOTUNE | (FLAG_PERSISTENT if persistent else 0)})
    ds.estimate(jobs, o)
    _check(ds, jobs, ref, f"table {table}")
    assert len(ctx.tune_table()) == len(table)  # every class was known: nothing re-tuned
    ds.close()
    ctx.close()


def test_autotuner_table_and_results(uneven):
    sc, opts, jobs, ref = uneven
    ctx = mvs.Context(0)
    ds = mvs.DeviceScene(sc.views, ctx)
    o = MvsOptions(**{**opts.__dict__, "flags": FLAG_AUTOTUNE | FLAG_PERSISTENT | FLAG_CUDA_GRAPH})
    ds.estimate(jobs, o)  # tunes the classes first
    _check(ds, jobs, ref, "autotuned")
    tab = ctx.tune_table()
    classes = {(sc.views[r].w, sc.views[r].h) for (r, _, _, _) in jobs}
    assert {(e["w"], e["h"]) for e in tab} == classes
    npx = {e["tile_w"] * e["tile_h"] for e in tab}
    assert len(npx) == 1 and npx.pop() in (32, 64, 128, 256)
    for e in tab:
        assert e["threads_per_pixel"] in (1, 5)
        assert 0 < e["ms_best"] <= e["ms_default"] or e["tile_w"] * e["tile_h"] != 64 or e["threads_per_pixel"] != 1
    # explicit call on known classes changes nothing
    assert ds.autotune(jobs, opts) == tab
    with pytest.raises(mvs.RcmvsError):
        ctx.set_tune_table([dict(w=96, h=72, tile_w=16, tile_h=20)])  # 320 pixels
    ds.close()
    ctx.close()


def test_learned_init_with_batched_schedules(uneven):
    sc, opts, jobs, ref = uneven
    ctx = mvs.Context(0)
    net = learned.ProposalNet(ctx, seed=5)
    a = mvs.DeviceScene(sc.views, ctx)
    b = mvs.DeviceScene(sc.views, ctx)
    na = learned.estimate_learned(a, jobs, opts, net, conf_thr=0.0)
    o = MvsOptions(**{**opts.__dict__, "flags": FLAG_PERSISTENT | FLAG_CUDA_GRAPH})
    for _ in range(2):
        nb = learned.estimate_learned(b, jobs, o, net, conf_thr=0.0)
        assert na == nb and na > 0
        for (r, _, _, _) in jobs:
            da, db = a.depth(r, normals=True), b.depth(r, normals=True)
            assert np.array_equal(bits(da.depth), bits(db.depth))
            assert np.array_equal(bits(da.cost), bits(db.cost))
            assert np.array_equal(bits(da.normal), bits(db.normal))
    a.close()
    b.close()
    net.close()
    ctx.close()


def test_scene_buffers_reused_across_scenes(uneven):
    """A context hands the buffers of a destroyed scene to the next scene
    that fits in them: results stay the oracle's whatever the sequence of
    scene sizes, and a context closed before its scene detaches it."""
    sc, opts, jobs, ref = uneven
    ctx = mvs.Context(0)
    big = mvs.DeviceScene(sc.views, ctx)
    big.estimate(jobs, opts)
    _check(big, jobs, ref, "first scene")
    big.close()
    # smaller scenes (the views one job touches) adopt the buffers, larger ones allocate
    for (r, srcs, a, b) in jobs[:3] + [jobs[0]]:
        sub = [r] + list(srcs)
        remap = {v: i for i, v in enumerate(sub)}
        views = [sc.views[v] for v in sub]
        dm = mvs.estimate_depth(views, 0, [remap[s] for s in srcs], a, b, opts, ctx, normals=True)
        d, c, n = ref[r]
        assert np.array_equal(bits(dm.depth), bits(d)) and np.array_equal(bits(dm.cost), bits(c))
        again = mvs.DeviceScene(sc.views, ctx)
        again.estimate(jobs, opts)
        _check(again, jobs, ref, "after a smaller scene")
        again.close()
    orphan = mvs.DeviceScene(sc.views, ctx)
    ctx.close()
    orphan.close()  # its context is gone: the scene frees its own buffers


# ---------------------------------------------- five lanes per pixel (passes)
@pytest.mark.parametrize("tile", [(8, 8), (16, 4), (8, 4), (16, 8), (32, 4)])
@pytest.mark.parametrize("flags", [0, FLAG_PERSISTENT, FLAG_PERSISTENT | FLAG_CUDA_GRAPH])
def test_split_passes_match_oracle(uneven, tile, flags):
    """threads_per_pixel 5 (one lane per window column, the row's counts
    exchanged by shuffles, source-independent depths kept across sources):
    the oracle's bits on the uneven batch (K 1-6, three sizes)."""
    sc, opts, jobs, ref = uneven
    ctx = mvs.Context(0)
    ds = mvs.DeviceScene(sc.views, ctx)
    o = MvsOptions(**{**opts.__dict__, "flags": flags, "tile_w": tile[0], "tile_h": tile[1], "threads_per_pixel": 5})
    ds.estimate(jobs, o)
    _check(ds, jobs, ref, f"split passes, tile {tile}, flags {flags}")
    ds.close()
    ctx.close()


def test_split_passes_count_the_same_work(uneven):
    """The work counters (plane_cost calls and 5-term rows) of the streamed
    passes (the default), the lockstep passes (one thread per pixel) and the
    split passes (five lanes per pixel) are equal, with and without the
    duplicate skip."""
    import os
    sc, opts, jobs, ref = uneven
    os.environ["RCMVS_COUNT"] = "1"
    try:
        ctx = mvs.Context(0)
    finally:
        del os.environ["RCMVS_COUNT"]
    ds = mvs.DeviceScene(sc.views, ctx)
    for flags in (0, 16):
        got = []
        for tpp, extra in ((1, 0), (1, FLAG_LOCKSTEP_PASSES), (5, 0)):
            ds.estimate(jobs, MvsOptions(**{**opts.__dict__, "flags": flags | extra, "threads_per_pixel": tpp}))
            got.append(ctx.last_work())
            _check(ds, jobs, ref, f"tpp {tpp} flags {flags | extra}")
        assert got[0] == got[1] == got[2] and got[0][0] > 0
    ds.close()
    ctx.close()


def test_split_passes_reject_bad_settings(uneven):
    sc, opts, jobs, _ = uneven
    ctx = mvs.Context(0)
    ds = mvs.DeviceScene(sc.views, ctx)
    for kw in (dict(threads_per_pixel=3), dict(threads_per_pixel=5, tile_w=16, tile_h=16)):
        with pytest.raises(mvs.RcmvsError):
            ds.estimate(jobs, MvsOptions(**{**opts.__dict__, **kw}))
    ds.close()
    ctx.close()
