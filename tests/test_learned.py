"""Learned plane proposals: CPU checks of the FP32 oracle and label
construction, GPU checks of the tensor-core network kernels against the
oracle, of the cost volume against a numpy restatement, and of the seeded
stereo."""
import numpy as np
import pytest

from oracle import net_oracle, oracle
from rustcolmap_b200 import MvsOptions, learned, mvs, scene


# ------------------------------------------------------------------ CPU
def test_param_layout_matches_library():
    assert learned.param_count() == net_oracle.param_layout()[1] == 55472


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    _, n = net_oracle.param_layout()
    p = (rng.normal(size=n) * 0.1).astype(np.float32)
    x = rng.uniform(size=(1, 5, 6, 48)).astype(np.float32)
    x[..., 33:] = 0
    lab = np.zeros((1, 5, 6, 8), np.float32)
    lab[..., 0] = rng.uniform(size=(1, 5, 6))
    nv = rng.normal(size=(1, 5, 6, 3))
    lab[..., 1:4] = nv / np.linalg.norm(nv, axis=-1, keepdims=True)
    lab[..., 4] = rng.uniform(size=(1, 5, 6)) > 0.3
    lab[..., 5] = 0.05
    loss, g = net_oracle.gradients(p, x, lab, bf=False)
    idx = np.nonzero(g)[0]
    idx = rng.choice(idx, 40, replace=False)
    ok = 0
    for i in idx:
        e = np.zeros(n, np.float32)
        e[i] = 1e-3
        fd = (net_oracle.gradients(p + e, x, lab, bf=False)[0] - net_oracle.gradients(p - e, x, lab, bf=False)[0]) / 2e-3
        ok += abs(fd - g[i]) <= 0.05 * abs(fd) + 2e-3
    assert ok >= 38  # a step may straddle a ReLU or |.| kink


def test_quarter_labels_of_a_plane():
    h, w = 16, 24
    depth = np.full((h, w), 4.0, np.float32)
    depth[:4, :4] = 0  # an empty block
    normal = np.zeros((h, w, 3), np.float32)
    normal[..., 2] = 1
    lab = learned.quarter_labels(depth, normal, 2.0, 8.0)
    imin, imax = learned.inv_range(2.0, 8.0)
    assert lab.shape == (4, 6, 8)
    assert lab[0, 0, 4] == 0 and (lab[..., 4].sum() == 23)
    assert np.allclose(lab[1, 1, 0], (0.25 - imin) / (imax - imin))
    assert np.allclose(lab[1, 1, 1:4], [0, 0, 1]) and np.allclose(lab[1, 1, 5], 0.02 * 0.25 / (imax - imin))


# ------------------------------------------------------------------ GPU
@pytest.fixture(scope="module")
def ctx():
    c = mvs.Context(0)
    yield c
    c.close()


def _random_batch(rng, n=2, h=20, w=37):
    x = rng.uniform(size=(n, h, w, 48)).astype(np.float32)
    x[..., 33:] = 0
    lab = np.zeros((n, h, w, 8), np.float32)
    lab[..., 0] = rng.uniform(size=(n, h, w))
    nv = rng.normal(size=(n, h, w, 3))
    lab[..., 1:4] = nv / np.linalg.norm(nv, axis=-1, keepdims=True)
    lab[..., 4] = rng.uniform(size=(n, h, w)) > 0.2
    lab[..., 5] = 0.05
    return net_oracle.bf16(x), lab


@pytest.mark.gpu
def test_net_forward_and_gradients_match_cpu_oracle(ctx):
    import torch
    rng = np.random.default_rng(1)
    net = learned.ProposalNet(ctx, seed=3)
    p = net.params()
    x, lab = _random_batch(rng)
    n, h, w = x.shape[:3]
    xd = torch.from_numpy(x).to(torch.bfloat16).cuda()
    ld = torch.from_numpy(lab).cuda()
    out = torch.empty((n, h, w, 16), dtype=torch.float32, device="cuda")
    net.forward(xd.data_ptr(), n, h, w, out.data_ptr())
    ctx.synchronize()
    acts, _, _ = net_oracle.forward(p, x)
    ref = acts[-1]
    got = out.cpu().numpy()
    assert np.abs(got - ref).max() <= 2e-2 * np.abs(ref).max()
    loss, g = net.train_step(xd.data_ptr(), ld.data_ptr(), n, h, w, 0.0, apply=False, grads=True)
    rloss, rg = net_oracle.gradients(p, x, lab)
    assert abs(loss - rloss) <= 1e-2 * abs(rloss)
    lay, _ = net_oracle.param_layout()
    for (wo, wn), (bo, bn), _, _ in lay:
        for a, b in ((g[wo:wo + wn], rg[wo:wo + wn]), (g[bo:bo + bn], rg[bo:bo + bn])):
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            assert cos > 0.995, cos
            assert np.linalg.norm(a - b) <= 0.06 * np.linalg.norm(b)
    net.close()


def _costvol_numpy(sc, ref, srcs, zmin, zmax):
    """numpy restatement of the cost volume (quarter resolution)."""
    def quarter(v):
        g = v.gray.astype(np.int64)
        hq, wq = v.h // 4, v.w // 4
        gq = ((g[: 4 * hq, : 4 * wq].reshape(hq, 4, wq, 4).sum((1, 3)) + 8) >> 4).astype(np.uint8)
        cam = ((v.cam.f / 4), (v.cam.cx - 1.5) / 4, (v.cam.cy - 1.5) / 4, v.cam.k)
        return gq, cam
    gr, cr = quarter(sc.views[ref])
    hq, wq = gr.shape
    cen = oracle.census_map(gr)
    xs, ys = np.meshgrid(np.arange(wq), np.arange(hq))
    rx = ((xs - cr[1]) / cr[0]).astype(np.float32)
    ry = ((ys - cr[2]) / cr[0]).astype(np.float32)
    imin, imax = learned.inv_range(zmin, zmax)
    out = np.zeros((hq, wq, 48), np.float32)
    srcd = []
    for s in srcs:
        gs, cs = quarter(sc.views[s])
        Rr, tr = sc.views[ref].R, sc.views[ref].t
        Rs, ts = sc.views[s].R, sc.views[s].t
        rs = (Rs @ Rr.T).astype(np.float32)
        tt = (ts - (Rs @ Rr.T) @ tr).astype(np.float32)
        srcd.append((oracle.census_map(gs), cs, rs, tt, gs.shape))
    for p in range(32):
        d = np.float32(1.0) / (imin + (imax - imin) * np.float32((p + 0.5) / 32))
        hs = np.zeros((hq, wq), np.int64)
        for ky in range(3):
            for kx in range(3):
                yy = np.clip(ys + ky - 1, 0, hq - 1)
                xx = np.clip(xs + kx - 1, 0, wq - 1)
                X = np.stack([d * rx[yy, xx], d * ry[yy, xx], np.full_like(rx, d)], -1)
                cref = cen[yy, xx]
                for cs_, cm, rs, tt, (sh, sw) in srcd:
                    P = X @ rs.T + tt
                    ok = P[..., 2] >= 1e-3
                    with np.errstate(all="ignore"):
                        u = np.trunc(cm[0] * P[..., 0] / P[..., 2] + cm[1])
                        v = np.trunc(cm[0] * P[..., 1] / P[..., 2] + cm[2])
                    ok &= (u >= 0) & (v >= 0) & (u < sw) & (v < sh)
                    ui = np.where(ok, u, 0).astype(np.int64)
                    vi = np.where(ok, v, 0).astype(np.int64)
                    x_ = cref ^ cs_[vi, ui]
                    pc = np.array([bin(int(q)).count("1") for q in x_.ravel()]).reshape(x_.shape)
                    hs += np.where(ok, pc, 48)
        out[..., p] = hs / (9 * 48 * len(srcs))
    out[..., 32] = gr / 255.0
    return out


@pytest.mark.gpu
def test_costvol_matches_numpy(ctx):
    import torch
    sc = scene.corner_room(seed=2, n_views=3, w=96, h=64, f=110.0, arc_deg=30.0, n_patches=20, per_view_sparse=60)
    ds = mvs.DeviceScene(sc.views, ctx)
    jobs = [(0, [1, 2], 2.5, 9.0)]
    out = torch.empty((16, 24, 48), dtype=torch.bfloat16, device="cuda")
    learned.costvol(ds, jobs, out.data_ptr())
    ctx.synchronize()
    got = out.float().cpu().numpy()
    ref = _costvol_numpy(sc, 0, [1, 2], 2.5, 9.0)
    assert np.array_equal(got[..., 33:], np.zeros_like(got[..., 33:]))
    assert np.allclose(got[..., 32], net_oracle.bf16(ref[..., 32]))
    diff = np.abs(got[..., :32] - ref[..., :32])
    assert diff.mean() < 2e-3 and (diff <= 1.0 / (9 * 48 * 2) + 4e-3).mean() > 0.99
    ds.close()


@pytest.mark.gpu
def test_learned_init_with_no_confident_pixel_equals_plain(ctx, corner_scene, c1_opts):
    v = corner_scene.views
    srcs, zr, _ = mvs.plan(corner_scene.sparse, v, c1_opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in (0, 4)]
    net = learned.ProposalNet(ctx, seed=1)
    a = mvs.DeviceScene(v, ctx)
    a.estimate(jobs, c1_opts)
    b = mvs.DeviceScene(v, ctx)
    assert learned.estimate_learned(b, jobs, c1_opts, net, conf_thr=2.0) == 0
    for j in jobs:
        da, db = a.depth(j[0], normals=True), b.depth(j[0], normals=True)
        assert np.array_equal(da.depth.view(np.uint32), db.depth.view(np.uint32))
        assert np.array_equal(da.cost.view(np.uint32), db.cost.view(np.uint32))
    # every confident, gate-passing pixel is seeded by the network
    n = learned.estimate_learned(b, jobs, c1_opts, net, conf_thr=0.0)
    assert 0 < n <= 2 * v[0].w * v[0].h
    a.close()
    b.close()
    net.close()


@pytest.mark.gpu
def test_training_reduces_loss(ctx):
    import torch
    sc = scene.orbit_room(seed=77, n_views=6, sizes=((160, 120),), n_boxes=6, per_view_sparse=100)
    opts = MvsOptions(max_dim=4096, num_sources=3, sweeps=2, num_hyp=32)
    srcs, zr, _ = mvs.plan(sc.sparse, sc.views, opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(6) if srcs[i]]
    ds = mvs.DeviceScene(sc.views, ctx)
    ds.estimate(jobs, opts)
    x = torch.empty((len(jobs), 30, 40, 48), dtype=torch.bfloat16, device="cuda")
    learned.costvol(ds, jobs, x.data_ptr())
    lab = np.stack([learned.quarter_labels(ds.depth(j[0], normals=True).depth, ds.depth(j[0], normals=True).normal,
                                           j[2], j[3]) for j in jobs])
    ld = torch.from_numpy(lab).cuda()
    net = learned.ProposalNet(ctx, seed=0)
    losses = learned.train(net, x, ld, iters=120, batch=len(jobs), lr=3e-3, log=None)
    assert np.mean(losses[-20:]) < 0.7 * np.mean(losses[:5])
    ds.close()
    net.close()


@pytest.mark.gpu
def test_run_mvs_learned_without_confident_pixels_equals_run_mvs(ctx, corner_scene, c1_opts):
    net = learned.ProposalNet(ctx, seed=2)
    _, xa, ca = mvs.run_mvs(corner_scene.views, corner_scene.sparse, c1_opts, ctx=ctx)
    _, xb, cb = mvs.run_mvs(corner_scene.views, corner_scene.sparse, c1_opts, ctx=ctx, net=net, conf_thr=2.0)
    assert np.array_equal(xa, xb) and np.array_equal(ca, cb)
    net.close()
