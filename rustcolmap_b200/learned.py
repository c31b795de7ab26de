"""Learned plane proposals that seed patch-match (no reference counterpart).

The network, its training step and the seeded stereo run in librcmvs
(include/rcmvs.h, "learned plane proposals"); this module drives them:
dataset generation (plain GPU patch-match depth maps of seeded synthetic
scenes as labels), training, evaluation against the plain method, and the
committed weights.

    python -m rustcolmap_b200.learned train --seeds 200 --out weights/proposal_c4.npy
    python -m rustcolmap_b200.learned eval  --weights weights/proposal_c4.npy --seeds 20
"""
import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import _abi, _lib, mvs, scene
from .types import MvsOptions

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "proposal_c4.npy")
COSTVOL_C, NET_OUT_C, LABEL_C = 48, 16, 8


def param_count():
    return int(_lib.mvs().rcmvs_net_param_count())


class ProposalNet:
    def __init__(self, ctx=None, params=None, seed=0):
        self.ctx = ctx or mvs.default_context()
        p = C.c_void_p()
        arr = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if arr is not None:
            assert arr.size == param_count()
        self.ctx.check(self.ctx._L.rcmvs_net_create(self.ctx.ptr, _abi.ptr(arr), int(seed), C.byref(p)))
        self.ptr = p

    def params(self):
        out = np.empty(param_count(), np.float32)
        self.ctx.check(self.ctx._L.rcmvs_net_get_params(self.ptr, out.ctypes.data))
        return out

    def forward(self, x, n, h, w, out):
        """x, out: device pointers (BF16 n*h*w*48 in, f32 n*h*w*16 out)."""
        self.ctx.check(self.ctx._L.rcmvs_net_forward(self.ctx.ptr, self.ptr, x, n, h, w, out))

    def train_step(self, x, labels, n, h, w, lr, apply=True, grads=False):
        loss = C.c_float()
        g = np.empty(param_count(), np.float32) if grads else None
        self.ctx.check(self.ctx._L.rcmvs_net_train_step(self.ctx.ptr, self.ptr, x, labels, n, h, w,
                                                        float(lr), int(bool(apply)), C.byref(loss),
                                                        _abi.ptr(g)))
        return (loss.value, g) if grads else loss.value

    def close(self):
        if getattr(self, "ptr", None):
            self.ctx._L.rcmvs_net_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _jobs_c(jobs):
    cj = (_abi.Job * len(jobs))()
    keep = []
    for i, (ref, srcs, zmin, zmax) in enumerate(jobs):
        s = np.ascontiguousarray(srcs, dtype=np.int32)
        keep.append(s)
        cj[i] = _abi.Job(int(ref), len(s), s.ctypes.data if len(s) else None, float(zmin), float(zmax))
    cj._keep = keep
    return cj


def costvol(ds, jobs, out_ptr):
    """Network input of every job (quarter resolution, back to back) into a
    device buffer of BF16 (sum_j (w_j/4)(h_j/4) * 48 elements)."""
    cj = _jobs_c(jobs)
    ds.ctx.check(ds.ctx._L.rcmvs_scene_costvol(ds.ctx.ptr, ds.ptr, cj, len(jobs), out_ptr))


# Operating point: the predicted plane alone for pixels with confidence >=
# 0.02, chosen on the tuning scenes (seeds 5000-5019) as the lowest threshold
# whose accuracy stays 1 point above the plain method with 6 sweeps, with no
# scene below it.  (A local sweep of 3 to 16 planes over +-1% to +-6% of the
# range around the prediction was both slower and less accurate.)
LOCAL_HYPS, LOCAL_SPAN, CONF_THR = 1, 0.0, 0.02
LEARNED_FLAGS = 0  # RCMVS_FLAG_* bits of the learned arm
# The learned arm's schedule and final gate: learned init + LEARNED_PASSES
# Jacobi passes (the passes option; the perturbations anneal over them), a
# pixel valid when its cost is below LEARNED_COST_THR.  Chosen on the tuning
# scenes (seeds 5000-5019) by a rule fixed before the held-out run: the
# fastest schedule whose coverage (pixels with ground truth valid and within
# 1%) and precision (valid pixels within 1%) both reach the plain method's
# with 6 sweeps at the reference's gate (0.38: 0.2532 / 0.842), at the gate
# with the largest smaller relative margin of the two.  With the committed
# weights (800 training scenes) 3 passes reach both at no gate (0.2548 /
# 0.841 at 0.255); 4 passes qualify at gates 0.24-0.26, and 0.245 gives
# 0.2595 / 0.862 (+2.5% / +2.4%).
LEARNED_PASSES, LEARNED_COST_THR = 4, 0.245
LEARNED_SWEEPS = 3  # sweeps field of the learned arm's options (passes overrides it)


def learned_options(opts):
    """opts with the learned arm's pass count, gate and flags."""
    import dataclasses
    return dataclasses.replace(opts, sweeps=LEARNED_SWEEPS, passes=LEARNED_PASSES, cost_thr=LEARNED_COST_THR,
                               flags=opts.flags | LEARNED_FLAGS)


def estimate_learned(ds, jobs, opts, net, conf_thr=CONF_THR, n_local=LOCAL_HYPS, span=LOCAL_SPAN):
    """Stereo seeded by the network; returns the number of learned-seeded pixels."""
    cj = _jobs_c(jobs)
    o = opts.to_c()
    n = C.c_uint64()
    ds.ctx.check(ds.ctx._L.rcmvs_scene_estimate_depth_learned(ds.ctx.ptr, ds.ptr, cj, len(jobs), C.byref(o),
                                                              net.ptr, float(conf_thr), int(n_local), float(span),
                                                              C.byref(n)))
    return n.value


def estimate_seeded(ds, jobs, opts, pred, conf_thr=CONF_THR, n_local=LOCAL_HYPS, span=LOCAL_SPAN):
    """Stereo seeded by caller-given proposals: pred holds each job's
    quarter-resolution (h/4, w/4, 16) f32 map, jobs back to back, as a numpy
    array (host) or a CUDA tensor (device).  Returns the number of seeded
    pixels."""
    cj = _jobs_c(jobs)
    o = opts.to_c()
    n = C.c_uint64()
    if isinstance(pred, np.ndarray):
        arr = np.ascontiguousarray(pred, dtype=np.float32)
        ptr, on_dev = arr.ctypes.data, 0
    else:
        assert pred.is_cuda and pred.is_contiguous() and str(pred.dtype) == "torch.float32"
        ptr, on_dev = pred.data_ptr(), 1
    ds.ctx.check(ds.ctx._L.rcmvs_scene_estimate_depth_seeded(ds.ctx.ptr, ds.ptr, cj, len(jobs), C.byref(o), ptr,
                                                             on_dev, float(conf_thr), int(n_local), float(span),
                                                             C.byref(n)))
    return n.value


def predict(ds, jobs, net):
    """The network's quarter-resolution predictions of every job (jobs whose
    reference views share one size), as a CUDA tensor (n, h/4, w/4, 16)."""
    import torch
    sizes = {(ds.views[j[0]].w, ds.views[j[0]].h) for j in jobs}
    assert len(sizes) == 1, "predict() takes jobs of one view size"
    w, h = sizes.pop()
    hq, wq = h // 4, w // 4
    x = torch.empty((len(jobs), hq, wq, COSTVOL_C), dtype=torch.bfloat16, device=f"cuda:{ds.ctx.device}")
    costvol(ds, jobs, x.data_ptr())
    out = torch.empty((len(jobs), hq, wq, NET_OUT_C), dtype=torch.float32, device=x.device)
    net.forward(x.data_ptr(), len(jobs), hq, wq, out.data_ptr())
    ds.ctx.synchronize()
    return out


def inv_range(zmin, zmax):
    """The kernels' f32 inverse-depth range of a job."""
    return np.float32(1.0) / np.float32(zmax), np.float32(1.0) / np.float32(zmin)


def quarter_labels(depth, normal, zmin, zmax, min_valid=8):
    """Labels at quarter resolution from a full-resolution depth/normal map:
    per 4x4 block with >= min_valid valid pixels, the mean inverse depth as a
    fraction t of the job's inverse-depth range, the mean normal, valid = 1
    and a tolerance on t equal to 2% of the block's inverse depth (the
    confidence target is "prediction within tolerance")."""
    h, w = depth.shape
    hq, wq = h // 4, w // 4
    d = depth[: 4 * hq, : 4 * wq].reshape(hq, 4, wq, 4).transpose(0, 2, 1, 3).reshape(hq, wq, 16)
    nrm = normal[: 4 * hq, : 4 * wq].reshape(hq, 4, wq, 4, 3).transpose(0, 2, 1, 3, 4).reshape(hq, wq, 16, 3)
    v = d > 0
    cnt = v.sum(-1)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.where(v, 1.0 / np.where(v, d, 1.0), 0.0).sum(-1) / np.maximum(cnt, 1)
        nm = (nrm * v[..., None]).sum(-2)
        nm /= np.maximum(np.linalg.norm(nm, axis=-1, keepdims=True), 1e-9)
    imin, imax = inv_range(zmin, zmax)
    span = float(imax - imin)
    lab = np.zeros((hq, wq, LABEL_C), np.float32)
    ok = cnt >= min_valid
    lab[..., 0] = (inv - float(imin)) / span
    lab[..., 1:4] = nm
    lab[..., 4] = ok
    lab[..., 5] = 0.02 * inv / span
    lab[~ok] = 0
    return lab


def orbit_c4(seed, device=0, normals=False):
    """Config 4's scenes: seeded room + 20 boxes, 16 views at 960x720 on a
    120-degree arc (8 degrees apart: on a full orbit, 22.5 degrees apart, the
    plain method's census costs rarely pass its 0.38 gate and it labels
    almost nothing)."""
    return scene.orbit_room(seed=seed, n_views=16, sizes=((960, 720),), f_rel=1.1, n_boxes=20, n_spheres=0,
                            device=device, per_view_sparse=300, arc_deg=120.0, normals=normals)


C4_OPTS = MvsOptions(max_dim=960, num_sources=4, sweeps=6, num_hyp=64)


def make_dataset(seeds, ctx, torch, dev, log=print, labels="plain"):
    """Cost volumes (device, BF16) and labels (device, f32) of every view of
    the given scenes.  labels "plain": from the plain GPU patch-match (6
    sweeps); "gt": from the rendered ground-truth depth and normals (the
    renderer's normals face the camera; a patch-match plane's normal n has
    n . ray > 0, so they are negated)."""
    xs, labs = [], []
    nvalid = 0.0
    t0 = time.time()
    for k, seed in enumerate(seeds):
        sc = orbit_c4(seed, normals=labels == "gt")
        srcs, zr, _ = mvs.plan(sc.sparse, sc.views, C4_OPTS)
        jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(sc.views)) if srcs[i]]
        ds = mvs.DeviceScene(sc.views, ctx)
        if labels == "plain":
            ds.estimate(jobs, C4_OPTS)
        else:
            ds.prepare()  # census and rays, which the cost volume reads
        hq, wq = sc.views[0].h // 4, sc.views[0].w // 4
        x = torch.empty((len(jobs), hq, wq, COSTVOL_C), dtype=torch.bfloat16, device=dev)
        costvol(ds, jobs, x.data_ptr())
        if labels == "gt":
            maps = [(sc.gt_depth[j[0]], -sc.gt_normal[j[0]]) for j in jobs]
        else:
            maps = [(lambda m: (m.depth, m.normal))(ds.depth(j[0], normals=True)) for j in jobs]
        lab = np.stack([quarter_labels(d, n, j[2], j[3]) for (d, n), j in zip(maps, jobs)])
        ds.close()
        xs.append(x)
        labs.append(torch.from_numpy(lab).to(dev))
        nvalid += float(lab[..., 4].mean())
        if log and (k % 20 == 0 or k == len(seeds) - 1):
            log(f"dataset: scene {k + 1}/{len(seeds)} ({time.time() - t0:.0f} s), "
                f"valid label fraction {nvalid / (k + 1):.3f}")
    ctx.synchronize()
    return torch.cat(xs), torch.cat(labs)


def train(net, x, lab, iters=1500, batch=16, lr=1e-3, seed=0, log=print):
    import torch
    n, h, w = x.shape[0], x.shape[1], x.shape[2]
    g = torch.Generator(device=x.device)
    g.manual_seed(seed)
    losses = []
    for it in range(iters):
        idx = torch.randint(0, n, (batch,), device=x.device, generator=g)
        xb = x.index_select(0, idx).contiguous()
        lb = lab.index_select(0, idx).contiguous()
        torch.cuda.synchronize()
        cur_lr = lr * (0.1 if it > 0.8 * iters else 1.0)
        loss = net.train_step(xb.data_ptr(), lb.data_ptr(), batch, h, w, cur_lr)
        losses.append(loss)
        if log and (it % 100 == 0 or it == iters - 1):
            log(f"train: iter {it} loss {np.mean(losses[-100:]):.4f}")
    return losses


def evaluate(net, seeds, ctx, conf_thr=CONF_THR, sweeps_learned=None, log=print, n_local=LOCAL_HYPS, span=LOCAL_SPAN,
             flags=None, cost_thr=None, passes_learned=None):
    """On held-out scenes: the plain method with 6 sweeps, the plain method
    with the learned arm's schedule (what the network's init replaces it
    with), and learned init + that schedule: `passes_learned` passes
    (default LEARNED_PASSES), or `sweeps_learned` sweeps when that is given
    alone.  Reports stereo views/s (CUDA
    events on the library stream, second of two runs) and ground truth: the
    fraction of pixels with ground truth that are valid and within 1%
    inverse depth ('within') and of valid pixels that are ('accuracy')."""
    import torch
    rows = []
    if passes_learned is None:
        passes_learned = LEARNED_PASSES if sweeps_learned is None else 0
    sweeps_learned = LEARNED_SWEEPS if sweeps_learned is None else sweeps_learned
    short = MvsOptions(max_dim=C4_OPTS.max_dim, num_sources=C4_OPTS.num_sources, sweeps=sweeps_learned,
                       num_hyp=C4_OPTS.num_hyp, passes=passes_learned)
    lopts = MvsOptions(max_dim=C4_OPTS.max_dim, num_sources=C4_OPTS.num_sources, sweeps=sweeps_learned,
                       num_hyp=C4_OPTS.num_hyp, flags=LEARNED_FLAGS if flags is None else flags,
                       cost_thr=LEARNED_COST_THR if cost_thr is None else cost_thr, passes=passes_learned)
    for seed in seeds:
        sc = orbit_c4(seed)
        srcs, zr, _ = mvs.plan(sc.sparse, sc.views, C4_OPTS)
        jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(sc.views)) if srcs[i]]
        ds = mvs.DeviceScene(sc.views, ctx)
        stream = torch.cuda.ExternalStream(ctx.stream)
        res = {}
        for name, o in (("plain6", C4_OPTS), ("plain_short", short), ("learned", lopts)):
            nl = 0
            for rep in range(2):  # the first run warms up
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ctx.synchronize()
                e0.record(stream)
                if name == "learned":
                    nl = estimate_learned(ds, jobs, o, net, conf_thr, n_local, span)
                else:
                    ds.estimate(jobs, o)
                e1.record(stream)
                ctx.synchronize()
            ms = e0.elapsed_time(e1)
            comp = [scene.gt_metrics(ds.depth(j[0]).depth, sc.gt_depth[j[0]]) for j in jobs]
            within = sum(m["within"] for m in comp)
            gt_px = sum(m["gt_pixels"] for m in comp)
            valid = sum(m["valid"] for m in comp)
            px = sum(sc.views[j[0]].w * sc.views[j[0]].h for j in jobs)
            res[name] = {"ms": ms, "views_per_s": len(jobs) / (ms / 1e3), "within": within / gt_px,
                         "accuracy": within / max(valid, 1), "learned_fraction": nl / px}
        ds.close()
        rows.append(res)
        if log:
            log(f"eval seed {seed}: " + " | ".join(
                f"{k} {v['views_per_s']:.1f} views/s within {v['within']:.4f} acc {v['accuracy']:.3f}"
                + (f" seeded {v['learned_fraction']:.2f}" if k == "learned" else "") for k, v in res.items()))
    agg = {}
    for name in rows[0]:
        agg[name] = {k: float(np.mean([r[name][k] for r in rows])) for k in rows[0][name]}
    agg["speedup_vs_plain6"] = agg["learned"]["views_per_s"] / agg["plain6"]["views_per_s"]
    agg["within_gain_vs_plain_short"] = agg["learned"]["within"] - agg["plain_short"]["within"]
    return agg, rows


def load_weights(path=DEFAULT_WEIGHTS):
    return np.load(path).astype(np.float32)


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--seeds", type=int, default=200)
    ap.add_argument("--seed0", type=int, default=1000)
    ap.add_argument("--iters", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--weights", default=DEFAULT_WEIGHTS)
    ap.add_argument("--conf", type=float, default=CONF_THR)
    ap.add_argument("--json", default=None)
    ap.add_argument("--local-hyps", type=int, default=LOCAL_HYPS)
    ap.add_argument("--local-span", type=float, default=LOCAL_SPAN)
    ap.add_argument("--labels", choices=["plain", "gt"], default="plain",
                    help="train on the plain method's depth maps or on the rendered ground truth")
    a = ap.parse_args()
    ctx = mvs.default_context()
    dev = torch.device("cuda:0")
    if a.cmd == "train":
        x, lab = make_dataset(list(range(a.seed0, a.seed0 + a.seeds)), ctx, torch, dev, labels=a.labels)
        net = ProposalNet(ctx, seed=0)
        t0 = time.time()
        losses = train(net, x, lab, iters=a.iters, batch=a.batch, lr=a.lr)
        print(f"train: {a.iters} iterations in {time.time() - t0:.1f} s")
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        np.save(a.out, net.params())
        if a.json:
            json.dump({"losses": losses[::10], "seeds": a.seeds, "iters": a.iters}, open(a.json, "w"))
    else:
        net = ProposalNet(ctx, params=load_weights(a.weights))
        agg, rows = evaluate(net, list(range(a.seed0, a.seed0 + a.seeds)), ctx, conf_thr=a.conf,
                             n_local=a.local_hyps, span=a.local_span)
        print(json.dumps(agg))
        if a.json:
            json.dump({"aggregate": agg, "per_seed": rows}, open(a.json, "w"))


if __name__ == "__main__":
    main()
