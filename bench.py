#!/usr/bin/env python
"""Benchmark of the dense-MVS hot path on B200 (one JSON line on rank 0).

Workload (default, --config c5): the full-scale synthetic scene — 100 views at
1920x1080 of a room + 60 boxes + 10 spheres, f = 1.15 x 1920, K = 10 support
views, 64 plane-sweep hypotheses, 6 sweeps (12 Jacobi passes), fusion with
>= 3 consistent views, 1% relative depth agreement and a 1 px reprojection
gate.  One step = census + rays, patch-match stereo for all 100 views, and
geometric-consistency fusion with voxel dedup (the PLY vertex records are
packed on the device).  Two arms run on the same scene: the reference's
schedule (plane-sweep init + 6 sweeps) and learned init (the committed
proposal network, rustcolmap_b200/weights/proposal_c4.npy) + 4 Jacobi passes
with a 0.245 cost gate (the operating point where its ground-truth coverage
and precision both reach the plain arm's); both
report the fraction of ground-truth pixels within 1% inverse depth.

value  depth maps/s of the learned arm with inputs resident in HBM
       (rcmvs_scene_* calls), timed with CUDA events on the library's stream,
       max over ranks; "plain" holds the reference-schedule arm.
e2e    the same metric through rcmvs_run_mvs_learned with pinned host
       buffers: host->device copy of every view's grey + colour image,
       device->host read of the fused cloud, inside the timed region.

--impl reference times the reference algorithm's CPU implementation (the
oracle port; the Rust reference cannot be built here) on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c5|c3|c2|c1|sfm]

--config sfm times the SfM front end instead: SIFT extraction of 48 RGB
1600x1200 images and exhaustive mutual matching of their 1128 pairs per
step, through the host-buffer API (its own metric, images/s).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FP32_NOMINAL_TOPS = 148 * 128 * 1.965e9 / 1e12  # SMs x FP32 lanes x max clock (ops/s, no FMA pairing)
# DRAM bytes (read + write) per reference pixel of one pass launch, from an
# ncu capture of the streamed pass kernel on 12 views at 1920x1080, K = 10
# (learned arm, pass 2: 2.573 GB read + 1.300 GB written over 24.88 Mpx),
# scaled to the measured workload's pixels for roofline.traffic.
PASS_DRAM_BYTES_PER_PX = (2572771000 + 1299575000) / (12 * 1920 * 1080)


def configs():
    from rustcolmap_b200 import MvsOptions
    return {
        "c5": dict(desc="100 views 1920x1080, room + 60 boxes + 10 spheres, f=1.15*1920, K=10, 64 hyps, "
                        "6 sweeps (12 passes); fusion min_consistent=3, depth_diff=0.01, reprojection <= 1 px",
                   scene=dict(n_views=100, sizes=((1920, 1080),), f_rel=1.15, n_boxes=60, n_spheres=10),
                   opts=MvsOptions(max_dim=1920, num_sources=10, sweeps=6, num_hyp=64, min_consistent=3,
                                   depth_diff=0.01, reproj_px=1.0)),
        "c3": dict(desc="48 views, widths {480,720,960,1440,1920} at 4:3 or 16:9 (seeded per view), room + 20 "
                        "boxes, f=1.1*long side, K ~ U{4..12} per view (seeded), 64 hyps, 6 sweeps (12 passes)",
                   scene=dict(n_views=48, sizes=((480, 360), (480, 270), (720, 540), (720, 405), (960, 720),
                                                 (960, 540), (1440, 1080), (1440, 810), (1920, 1440),
                                                 (1920, 1080)),
                              f_rel=1.1, n_boxes=20, n_spheres=0, size_choice="random"),
                   k_range=(4, 12),
                   opts=MvsOptions(max_dim=1920, num_sources=12, sweeps=6, num_hyp=64)),
        "c2": dict(desc="64 views 960x720, room + 20 boxes, f=1.1*960, K=8, 64 hyps, 6 sweeps (12 passes)",
                   scene=dict(n_views=64, sizes=((960, 720),), f_rel=1.1, n_boxes=20, n_spheres=0),
                   opts=MvsOptions(max_dim=960, num_sources=8, sweeps=6, num_hyp=64)),
        "c1": dict(desc="corner room, 8 views 384x288, f=440, K=4, 64 hyps, 6 sweeps (12 passes)",
                   scene=None, opts=MvsOptions(max_dim=384, num_sources=4, sweeps=6, num_hyp=64)),
    }


def make_jobs(cfg, sc, opts, planner=None):
    """(ref, sources, zmin, zmax) per view with sources; with k_range each
    view keeps the first K ~ U{lo..hi} (seeded) of its planned sources.
    planner: the plan glue to use (default the library's rcmvs_plan)."""
    if planner is None:
        from rustcolmap_b200 import mvs
        planner = mvs.plan
    srcs, zr, fus = planner(sc.sparse, sc.views, opts)
    if "k_range" in cfg:
        rng = np.random.default_rng(3)
        lo, hi = cfg["k_range"]
        srcs = [s[:int(rng.integers(lo, hi + 1))] for s in srcs]
    return [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(sc.views)) if srcs[i]], fus


def make_scene(cfg, seed, device):
    from rustcolmap_b200 import scene
    if cfg["scene"] is None:
        return scene.corner_room(seed=seed, device=device)
    return scene.orbit_room(seed=seed, device=device, per_view_sparse=300, **cfg["scene"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(rows[0][2]),
                "power_w_max": max((num(r[3]) or 0) for r in rows), "samples": len(rows), "reasons": reasons}


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws, local):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, ws, local):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def pinned_views(views):
    """Copies of the views whose grey/colour images live in pinned host memory."""
    import copy

    import torch
    out = []
    for v in views:
        g = torch.empty(v.gray.shape, dtype=torch.uint8, pin_memory=True).numpy()
        g[...] = v.gray
        c = torch.empty(v.rgb.shape, dtype=torch.uint8, pin_memory=True).numpy()
        c[...] = v.rgb
        nv = copy.copy(v)
        nv.gray, nv.rgb = g, c
        out.append(nv)
    return out


def cpu_rows(args):
    """Rows of the CPU band: --cpu-rows, else sixteen per host thread (the
    oracle threads over rows, so every thread gets work and the rows' uneven
    costs even out; at 1920 wide, K=10, 12 passes that is about 10 s of CPU
    work per sample)."""
    return args.cpu_rows or 16 * (os.cpu_count() or 1)


def cpu_baseline(sc, opts, jobs, rows, threads=0):
    """Times the oracle's estimate_depth on a band of `rows` rows of the first
    job's reference view (a bounded sample of one view; stereo only, the
    fusion is not part of the sample).  Returns (depth maps/s, seconds,
    sample description, threads)."""
    import copy

    from oracle import oracle
    ref, srcs, zmin, zmax = jobs[0]
    v = sc.views[ref]
    y0 = max(0, v.h // 2 - rows // 2)
    band = copy.copy(v)
    band.gray = np.ascontiguousarray(v.gray[y0:y0 + rows])
    band.h = band.gray.shape[0]
    band.cam = type(v.cam)(v.cam.f, v.cam.cx, v.cam.cy - y0, v.cam.k)
    views = list(sc.views)
    views[ref] = band
    nt = threads or os.cpu_count() or 1
    t0 = time.perf_counter()
    oracle.estimate_depth(views, ref, srcs, zmin, zmax, opts, nthreads=nt, normals=False)
    dt = time.perf_counter() - t0
    frac = band.h / v.h
    desc = (f"oracle estimate_depth on a {v.w}x{band.h} band (rows {y0}-{y0 + band.h}) of one "
            f"{v.w}x{v.h} view, K={len(srcs)}, {opts.num_hyp} hyps, {2 * opts.sweeps} passes, {nt} threads; "
            f"{frac:.4f} of a depth map per sample; stereo only (fusion not sampled)")
    return frac / dt, dt, desc, nt


def run_reference(args, cfg):
    """The reference algorithm's CPU implementation (the oracle port) on the
    host cores, rank 0 only.  Loads no library of the product: the scene is
    rendered by the host-only build of the renderer (oracle/libscene_host.so)
    and planned by the oracle's plan glue."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    from rustcolmap_b200 import scene
    oracle.lib()
    scene.use_host_renderer(os.path.join(ROOT, "oracle", "libscene_host.so"))
    t_setup = time.perf_counter()
    sc = make_scene(cfg, seed=5, device=-1)
    opts = cfg["opts"]
    jobs, fus = make_jobs(cfg, sc, opts, planner=oracle.plan)
    setup_s = time.perf_counter() - t_setup
    rows = cpu_rows(args)
    for _ in range(args.warmup):
        cpu_baseline(sc, opts, jobs, rows)
    times, rate, desc, nt = [], 0.0, "", 0
    for _ in range(args.steps):
        r, dt, desc, nt = cpu_baseline(sc, opts, jobs, rows)
        times.append(dt)
    frac = min(rows, sc.views[jobs[0][0]].h) / sc.views[jobs[0][0]].h
    rate = frac * len(times) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "depth maps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": args.config + ": " + cfg["desc"], "setup_s": setup_s,
                                            "inputs": "scene rendered on the host (oracle/libscene_host.so), "
                                                      "plan by the oracle (orc_plan)"},
            "cpu_baseline": {"value": rate, "unit": "depth maps/s", "cores": nt, "kind": "port",
                             "sample": desc},
            "e2e": {"value": rate, "unit": "depth maps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


METRIC = "1080p depth maps/s at K=10: learned-init vs plain GPU patch-match at equal GT error"


def gt_summary(ds, sc, jobs, scene, stricter_gate=None):
    """Ground truth over every job: fraction of pixels with ground truth that
    are valid and within 1% inverse depth ('within_1pct', coverage), and the
    same over valid pixels ('accuracy', precision).  With stricter_gate the
    same two figures are added for the maps gated at that cost (a stricter
    gate only removes pixels, so the run's own maps give them).  'fused':
    the fused cloud's distances to the scene's analytic surfaces."""
    within = gt_px = valid = 0
    w2 = v2 = 0
    for (ref, _, _, _) in jobs:
        dm = ds.depth(ref)
        m = scene.gt_metrics(dm.depth, sc.gt_depth[ref])
        within += m["within"]
        gt_px += m["gt_pixels"]
        valid += m["valid"]
        if stricter_gate is not None:
            m2 = scene.gt_metrics(np.where(dm.cost < stricter_gate, dm.depth, 0).astype(np.float32), sc.gt_depth[ref])
            w2 += m2["within"]
            v2 += m2["valid"]
    out = {"within_1pct": within / max(gt_px, 1), "accuracy": within / max(valid, 1),
           "tol": "1% relative inverse depth", "views": len(jobs)}
    if stricter_gate is not None:
        out[f"at_gate_{stricter_gate:g}"] = {"within_1pct": w2 / max(gt_px, 1), "accuracy": w2 / max(v2, 1)}
    if getattr(sc, "prims", None) and ds.n_points:
        # fused cloud against the analytic surfaces (scene units; the room is 12 x 12 x 4)
        d = scene.surface_distance(ds.points()[0], sc.prims)
        out["fused"] = {"points": int(len(d)), "median_dist": float(np.median(d)),
                        "mean_dist": float(d.mean()), "within_0.01": float((d <= 0.01).mean()),
                        "within_0.02": float((d <= 0.02).mean()), "unit": "scene units"}
    return out


SFM_METRIC = "1600x1200 images/s through SIFT (2048 features) + exhaustive mutual matching of all pairs"
SFM_IMAGES = 48
SFM_DESC = (f"{SFM_IMAGES} synthetic RGB views 1600x1200 (room + 20 boxes, orbit); step = extract_sift on every "
            f"view (max_dim 1600, 2048 features, contrast 0.0067) + match_pair on all "
            f"{SFM_IMAGES * (SFM_IMAGES - 1) // 2} pairs (ratio 0.8)")


def sfm_images(device):
    from rustcolmap_b200 import scene
    sc = scene.orbit_room(seed=11, n_views=SFM_IMAGES, sizes=((1600, 1200),), n_boxes=20, per_view_sparse=10,
                          device=device)
    return [np.ascontiguousarray(v.rgb) for v in sc.views]


def sfm_cpu(imgs, n_img, n_pairs):
    """The oracle on all host cores: SIFT on n_img images and match_pair on
    n_pairs pairs of their descriptors, images and pairs spread over a
    thread pool (the oracle's C calls release the GIL).  Returns (images/s
    of the full step composition, sample description, threads)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle
    from rustcolmap_b200 import colmap
    nt = os.cpu_count() or 1
    preps = [colmap.gray_rgb(im) for im in imgs[:n_img]]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(nt) as ex:
        outs = list(ex.map(lambda p: oracle.extract_sift(p[0], p[1]), preps))
    t_img = (time.perf_counter() - t0) / n_img
    descs = [o[1] for o in outs]
    prs = [(i % n_img, (i + 1 + i // n_img) % n_img) for i in range(n_pairs)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(nt) as ex:
        list(ex.map(lambda q: oracle.match_pair(descs[q[0]], descs[q[1]]), prs))
    t_pair = (time.perf_counter() - t0) / n_pairs
    step = SFM_IMAGES * t_img + SFM_IMAGES * (SFM_IMAGES - 1) // 2 * t_pair
    desc = (f"{n_img} images and {n_pairs} pairs on {nt} threads ({1e3 * t_img:.0f} ms per image, "
            f"{1e3 * t_pair:.1f} ms per pair, amortised), scaled to the step's {SFM_IMAGES} images and "
            f"{SFM_IMAGES * (SFM_IMAGES - 1) // 2} pairs")
    return SFM_IMAGES / step, desc, nt


def run_sfm(args):
    """--config sfm: the SfM front end (SIFT + matching) on one GPU."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        from rustcolmap_b200 import scene
        scene.use_host_renderer(os.path.join(ROOT, "oracle", "libscene_host.so"))
        imgs = sfm_images(-1)
        for _ in range(args.warmup):
            sfm_cpu(imgs, 2, 4)
        vals = [sfm_cpu(imgs, 16, 48) for _ in range(args.steps)]
        v = statistics.median(x[0] for x in vals)
        line = {"impl": "reference", "metric": SFM_METRIC, "value": v, "unit": "images/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * SFM_IMAGES / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
                "data": "synthetic", "config": {"workload": "sfm: " + SFM_DESC},
                "cpu_baseline": {"value": v, "unit": "images/s", "cores": vals[0][2], "kind": "port",
                                 "sample": vals[0][1]},
                "e2e": {"value": v, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch

    from rustcolmap_b200 import mvs, sift
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    imgs = sfm_images(local)
    ctx = mvs.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    pairs = [(i, j) for i in range(SFM_IMAGES) for j in range(i + 1, SFM_IMAGES)]
    state = {}
    # SIFT of the images spread over `sift_workers` contexts (one CUDA stream
    # and one host thread each, sift.extract_sift_many); matching on the
    # first context.  Extraction returns with its results on the host, so
    # the events on the first context's stream span the whole step.
    nw = max(1, args.sift_workers)
    ctxs = [ctx] + [mvs.Context(local) for _ in range(nw - 1)]

    def step():
        frames = sift.extract_sift_many(imgs, ctxs=ctxs)
        m = sift.match_pairs([f.desc for f in frames], pairs, 0.8, ctx)
        state.update(frames=frames, matches=m)

    for _ in range(args.warmup):
        step()
    clk = ClockSampler(local)
    for c in ctxs:
        c.timing(True)
    max_over_ranks(0.0, ws, local)
    torch.cuda.synchronize()
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms, ws, local)
    kt = {}
    for k in ("sift_pyramid", "sift_extrema", "sift_orient", "sift_desc", "match_dist", "match_select"):
        per = [c.kernel_time(k) for c in ctxs]  # summed over the contexts' streams
        kt[k] = (sum(p[0] for p in per), sum(p[1] for p in per))
    for c in ctxs:
        c.timing(False)
    frames, m = state["frames"], state["matches"]
    nfeat = [len(f.pts) for f in frames]
    ops = sum(nfeat[i] * nfeat[j] for i, j in pairs) * 128 * 3  # sub, mul, add per component
    dist_ms, dist_n = kt["match_dist"]
    dist_launch_ms = dist_ms / max(dist_n, 1)
    ops_per_launch = ops * args.steps / max(dist_n, 1)
    achieved = ops_per_launch / (dist_launch_ms * 1e-3) / 1e12
    value = ws * SFM_IMAGES / (ms * 1e-3)
    h2d = sum(im.nbytes for im in imgs) + sum(f.desc.nbytes for f in frames)
    d2h = sum(f.pts.nbytes + f.desc.nbytes + f.colors.nbytes for f in frames) + sum(a.nbytes + b.nbytes for a, b in m)
    line = {"metric": SFM_METRIC, "value": value, "unit": "images/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64 (SIFT), f32 (matching)", "data": "synthetic",
            "config": {"workload": "sfm: " + SFM_DESC, "l2": "inputs larger than L2 (276 MB of images)",
                       "sift_workers": nw,
                       "features_mean": float(np.mean(nfeat)),
                       "matches_mean": float(np.mean([len(a) for a, _ in m]))},
            "roofline": {"bound": "fp32_issue", "kernel": "match_dist", "achieved": achieved,
                         "peak": FP32_NOMINAL_TOPS, "unit": "Top/s", "frac": achieved / FP32_NOMINAL_TOPS,
                         "traffic": None, "peak_source": "nominal 148 SM x 128 FP32 lanes x 1.965 GHz",
                         "ops_per_launch": ops_per_launch, "avg_launch_ms": dist_launch_ms},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kt.items()},
            "e2e": {"value": value, "unit": "images/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "note": "value itself is measured through the host-buffer API (rcmvs_extract_sift, "
                            "rcmvs_match_pairs), copies included"},
            "clocks": clocks}
    if rank == 0 and not args.no_cpu_baseline:
        v, desc, nt = sfm_cpu(imgs, 16, 48)
        line["cpu_baseline"] = {"value": v, "unit": "images/s", "cores": nt, "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_shard(args, cfg):
    """--shard: ONE scene split over the N ranks (strong scaling): each rank
    runs stereo (the learned arm's schedule) for its share of the reference
    views, the depth maps and fusion candidates move device to device
    through NCCL, and every rank dedups the same candidate list
    (shard.run_mvs_sharded_device).  A step is the whole scene; value =
    depth maps of the scene per second, max over ranks."""
    import dataclasses
    import datetime

    import torch
    import torch.distributed as dist

    from rustcolmap_b200 import learned, mvs, shard
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:  # one rank: the same collectives on a group of one
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    opts = learned.learned_options(cfg["opts"])
    sc = make_scene(cfg, seed=5, device=local)  # the same scene on every rank
    n_maps = len(make_jobs(cfg, sc, opts)[0])
    ctx = mvs.Context(local)
    net = learned.ProposalNet(ctx, params=learned.load_weights())
    ops = shard.SceneOps(sc.views, opts, ctx, net=net)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    out = {}

    def step():
        out["xyz"], out["rgb"], _ = shard.run_mvs_sharded_device(sc.views, sc.sparse, opts, ops=ops,
                                                                  device=f"cuda:{local}")

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    ctx.synchronize()
    torch.cuda.synchronize()
    e1.record(stream)  # every stream of the step has drained before this
    e1.synchronize()
    dist.barrier()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), ws, local) / args.steps
    value = n_maps / (ms / 1e3)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "depth maps/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32 (stereo), bf16/f32-acc (proposal net)", "data": "synthetic",
                "config": {"workload": args.config + ": " + cfg["desc"], "views_per_step": n_maps,
                           "parallelism": f"one scene sharded over {ws} rank(s): reference views by "
                                         "longest-processing-time, depth maps and candidates all-gathered "
                                         "device to device (NCCL)",
                           "headline_arm": f"learned init (proposal_c4 weights) + {opts.sweeps} sweeps, "
                                           f"gate cost < {opts.cost_thr:g}"},
                "fused_points": int(len(out["xyz"])),
                "gpu_launches": args.steps * (1 + 3 + 6 + 1 + 2 * opts.sweeps + 1 + 5), "clocks": clocks}
        print(json.dumps(line), flush=True)
    ops.close()
    net.close()
    ctx.close()
    dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--sift-workers", type=int, default=4,
                    help="--config sfm: contexts (streams + host threads) the images' SIFT is spread over")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=["c5", "c3", "c2", "c1", "sfm"])
    ap.add_argument("--cpu-rows", type=int, default=0,
                    help="rows of the CPU band (cpu_baseline and --impl reference; default 16 per host thread)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--views", type=int, default=0, help="override the number of views (profiling runs)")
    ap.add_argument("--arc-deg", type=float, default=0.0,
                    help="cameras on an arc of this many degrees instead of the full orbit (profiling runs with "
                         "fewer views at the full scene's camera spacing)")
    ap.add_argument("--no-count", action="store_true", help="skip the work-counting rerun")
    ap.add_argument("--one-candidate", action="store_true",
                    help="use the one-candidate-at-a-time init kernel (comparison)")
    ap.add_argument("--plain-only", action="store_true", help="time only the plain (reference-schedule) arm")
    ap.add_argument("--learned-only", action="store_true", help="time only the learned arm (tuning runs)")
    ap.add_argument("--local-hyps", type=int, default=None)
    ap.add_argument("--local-span", type=float, default=None)
    ap.add_argument("--conf", type=float, default=None)
    ap.add_argument("--flags", type=int, default=0,
                    help="RCMVS_FLAG_* bits for both arms (2 persistent queue, 4 CUDA graph, 8 autotuned tiles)")
    ap.add_argument("--tile", default="", help="WxH stereo tile (default: the library's 8x8)")
    ap.add_argument("--tpp", type=int, default=0, help="threads per pixel of the Jacobi passes (1 or 5)")
    ap.add_argument("--shard", action="store_true",
                    help="one scene split over the --gpus ranks (strong scaling; device-to-device exchanges)")
    args = ap.parse_args()
    assert args.warmup >= 3 or os.environ.get("RCMVS_BENCH_ALLOW_SHORT"), "warm-up must be >= 3 steps"
    if args.config == "sfm":
        run_sfm(args)
        return
    cfg = configs()[args.config]
    if args.views and cfg["scene"] is not None:
        cfg["scene"] = dict(cfg["scene"], n_views=args.views)
        cfg["desc"] += f" [{args.views} views]"
    if args.arc_deg and cfg["scene"] is not None:
        cfg["scene"] = dict(cfg["scene"], arc_deg=args.arc_deg)
        cfg["desc"] += f" [{args.arc_deg:g} degree arc]"
    if args.impl == "reference":
        run_reference(args, cfg)
        return
    if args.shard:
        run_shard(args, cfg)
        return

    import dataclasses

    import torch

    from rustcolmap_b200 import learned, mvs, scene
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    opts = cfg["opts"]
    if args.one_candidate:
        opts.flags |= 1
    opts.flags |= args.flags
    if args.tile:
        opts.tile_w, opts.tile_h = map(int, args.tile.lower().split("x"))
    opts.threads_per_pixel = args.tpp
    lopts = learned.learned_options(opts)
    t_setup = time.perf_counter()
    sc = make_scene(cfg, seed=5 + 1000 * rank, device=local)
    jobs, fus = make_jobs(cfg, sc, opts)
    n_maps = len(jobs)
    ctx = mvs.Context(local)
    ds = mvs.DeviceScene(sc.views, ctx)
    net = None if args.plain_only else learned.ProposalNet(ctx, params=learned.load_weights())
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    setup_s = time.perf_counter() - t_setup
    seeded = [0]

    def step_plain():
        ds.prepare()
        ds.estimate(jobs, opts)
        return ds.fuse(fus, sc.sparse.xyz, opts)

    lkw = {}
    if args.local_hyps is not None:
        lkw["n_local"] = args.local_hyps
    if args.local_span is not None:
        lkw["span"] = args.local_span
    if args.conf is not None:
        lkw["conf_thr"] = args.conf

    def step_learned():
        ds.prepare()
        seeded[0] = learned.estimate_learned(ds, jobs, lopts, net, **lkw)
        return ds.fuse(fus, sc.sparse.xyz, lopts)

    def timed(step, clocks=False):
        for _ in range(args.warmup):
            step()
        ctx.synchronize()
        barrier(ws)
        clk = ClockSampler(local)
        if clocks:
            clk.start()
        ctx.timing(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        barrier(ws)
        e0.record(stream)
        npts = 0
        for _ in range(args.steps):
            npts = step()
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        barrier(ws)
        ck = clk.stop() if clocks else None
        ms = e0.elapsed_time(e1)
        names = ("census_rays", "learned_costvol", "learned_net", "learned_init", "stereo_init", "stereo_pass",
                 "stereo_gate", "fuse_candidates", "fuse_reduce")
        kt = {k: ctx.kernel_time(k) for k in names}
        ctx.timing(False)
        ms_max = max_over_ranks(ms, ws, local)
        gate = lopts.cost_thr if step is step_plain and lopts.cost_thr < opts.cost_thr else None
        return ms_max, kt, npts, ck, gt_summary(ds, sc, jobs, scene, stricter_gate=gate)

    if args.learned_only:  # tuning runs: no plain arm
        plain_ms, plain_kt, plain_pts, plain_clk, plain_gt = float("nan"), {}, 0, None, {"within_1pct": float("nan")}
    else:
        plain_ms, plain_kt, plain_pts, plain_clk, plain_gt = timed(step_plain, clocks=args.plain_only)
    if args.plain_only:
        head_ms, head_kt, head_pts, clocks, head_gt = plain_ms, plain_kt, plain_pts, plain_clk, plain_gt
    else:
        head_ms, head_kt, head_pts, clocks, head_gt = timed(step_learned, clocks=True)
    total_maps = sum_over_ranks(n_maps * args.steps, ws, local)
    value = total_maps / (head_ms / 1e3)
    plain_value = total_maps / (plain_ms / 1e3)
    head_opts = opts if args.plain_only else lopts

    # work counters of the plain arm (untimed rerun with counting on)
    # (and again with the duplicate skip off: the reference's own call count)
    evals, rows5, ref_evals, ref_rows5 = 0, 0, 0, 0
    if not args.no_count:
        os.environ["RCMVS_COUNT"] = "1"
        cctx = mvs.Context(local)
        del os.environ["RCMVS_COUNT"]
        cds = mvs.DeviceScene(sc.views, cctx)
        cds.estimate(jobs, opts)
        evals, rows5 = cctx.last_work()
        cds.estimate(jobs, dataclasses.replace(opts, flags=opts.flags | 16))
        ref_evals, ref_rows5 = cctx.last_work()
        cds.close()
        cctx.close()

    # end to end through the reference-facing call with pinned host buffers
    e2e = None
    if not args.no_e2e:
        pv = pinned_views(sc.views)
        for _ in range(max(args.warmup, 1)):  # warm: the first calls settle the context's buffers
            mvs.run_mvs(pv, sc.sparse, head_opts, ctx=ctx, net=net, **lkw)
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            st, xyz, rgb = mvs.run_mvs(pv, sc.sparse, head_opts, ctx=ctx, net=net, **lkw)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        barrier(ws)
        dt = max_over_ranks(dt, ws, local)
        h2d = int(sum(v.gray.nbytes + v.rgb.nbytes for v in pv))
        e2e = {"value": sum_over_ranks(n_maps * args.steps, ws, local) / dt, "unit": "depth maps/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(xyz.nbytes + rgb.nbytes),
               "ms_per_step": 1e3 * dt / args.steps, "call": "rcmvs_run_mvs" + ("" if net is None else "_learned"),
               # device spans of the call's stereo and fusion (CUDA events inside the call), last step
               "device_ms": {"stereo": 1e3 * st.stereo_s, "fuse": 1e3 * st.fuse_s}}

    # roofline of the dominant kernel (the Jacobi pass) in the headline arm
    npx = sum(sc.views[r].w * sc.views[r].h for r, _, _, _ in jobs)
    src_px = sum(sc.views[s].w * sc.views[s].h for _, ss, _, _ in jobs for s in ss)
    pass_ms, pass_n = head_kt["stereo_pass"]
    pass_avg_s = pass_ms / max(pass_n, 1) / 1e3
    bytes_per_launch = npx * (20 + 20 + 8 + 8) + src_px * 8
    achieved_gbs = bytes_per_launch / pass_avg_s / 1e9
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    algo_terms_total = sum(sc.views[r].w * sc.views[r].h * 25 * len(s) * (opts.num_hyp + 7 * 2 * opts.sweeps)
                           for r, s, _, _ in jobs)
    actual_terms = rows5 * 5
    stereo_ms = sum(plain_kt[k][0] for k in ("stereo_init", "stereo_pass", "stereo_gate")) / args.steps if plain_kt else 0
    fp32_ops_per_term = 40
    achieved_tops = actual_terms * fp32_ops_per_term / (stereo_ms / 1e3) / 1e12 if actual_terms and stereo_ms else None
    ref_tops = ref_rows5 * 5 * fp32_ops_per_term / (stereo_ms / 1e3) / 1e12 if ref_rows5 and stereo_ms else None

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and ws == 1:
        rate, dt, desc, nt = cpu_baseline(sc, opts, jobs, cpu_rows(args))
        cpu = {"value": rate, "unit": "depth maps/s", "cores": nt, "kind": "port", "sample": desc, "seconds": dt}
        # the same port on one thread, on a smaller band (a few seconds)
        rate1, dt1, desc1, _ = cpu_baseline(sc, opts, jobs, 4, threads=1)
        cpu["single_thread"] = {"value": rate1, "unit": "depth maps/s", "cores": 1, "sample": desc1,
                                "seconds": dt1}

    if rank == 0:
        n_pass = lambda o: o.passes if o.passes else 2 * max(o.sweeps, 1)
        per_step = (1 + 1 + n_pass(opts) + 1 + 5) if args.plain_only else (1 + 3 + 6 + 1 + n_pass(lopts) + 1 + 5)
        line = {
            "metric": METRIC, "value": value, "unit": "depth maps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (stereo), bf16/f32-acc (proposal net)",
            "data": "synthetic",
            "config": {"workload": args.config + ": " + cfg["desc"], "views_per_step": n_maps,
                       "headline_arm": "plain, 6 sweeps" if args.plain_only else
                       f"learned init (proposal_c4 weights; pixels with confidence >= "
                       f"{args.conf if args.conf is not None else learned.CONF_THR} start from the "
                       f"predicted plane, the others from the 64-plane sweep) + {n_pass(lopts)} passes, "
                       f"gate cost < {lopts.cost_thr:g}",
                       "parallelism": f"views batched on 1 GPU; {ws} rank(s), one independent scene each",
                       "l2": "inputs larger than L2 (census 8 B/px, rays 8 B/px, planes 40 B/px over all views)"},
            "plain": {"value": plain_value, "unit": "depth maps/s", "sweeps": opts.sweeps,
                      "ms_per_step": plain_ms / args.steps, "gt": plain_gt, "fused_points": plain_pts,
                      "kernel_ms_per_step": {k: v[0] / args.steps for k, v in plain_kt.items() if v[1]}},
            "learned": None if args.plain_only else {
                "value": value, "passes": n_pass(lopts), "gt": head_gt, "fused_points": head_pts,
                "seeded_fraction": seeded[0] / max(npx, 1), "speedup_vs_plain": value / plain_value,
                "gt_within_delta_vs_plain": head_gt["within_1pct"] - plain_gt["within_1pct"]},
            "roofline": {"bound": "hbm", "kernel": "stereo_pass", "achieved": achieved_gbs, "peak": hbm_peak,
                         "unit": "GB/s", "frac": achieved_gbs / hbm_peak,
                         "traffic": PASS_DRAM_BYTES_PER_PX * npx,
                         "traffic_source": "ncu dram bytes per pixel of a 12-view 1920x1080 K=10 capture of "
                                           "the streamed pass kernel (learned arm) x this launch's pixels",
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650",
                         "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": pass_avg_s * 1e3,
                         "note": "issue-bound kernel: see compute_roofline"},
            "compute_roofline": {"bound": "fp32_issue", "kernel": "stereo init + pass (plain arm)",
                                 "achieved": achieved_tops, "peak": FP32_NOMINAL_TOPS, "unit": "Top/s",
                                 "frac": achieved_tops / FP32_NOMINAL_TOPS if achieved_tops else None,
                                 "ops_per_term": fp32_ops_per_term,
                                 "peak_source": "nominal 148 SM x 128 FP32 lanes x 1.965 GHz",
                                 "note": "achieved counts the terms evaluated; reference_equivalent counts the "
                                         "terms the reference's call sequence evaluates for the same step "
                                         "(duplicate skip off), over the same time",
                                 "reference_equivalent": ref_tops,
                                 "reference_equivalent_frac": ref_tops / FP32_NOMINAL_TOPS if ref_tops else None},
            "gpu_launches": args.steps * per_step,
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gcost_evals_per_s_plain": evals * args.steps / (plain_ms / 1e3) / 1e9 if evals else None,
            "gcost_evals_per_s_plain_reference_equivalent":
                ref_evals * args.steps / (plain_ms / 1e3) / 1e9 if ref_evals else None,
            "work_plain": {"cost_evals_per_step": evals, "window_rows_per_step": rows5,
                           "algorithmic_cost_evals_per_step": sum(sc.views[r].w * sc.views[r].h *
                                                                 (opts.num_hyp + 14 * opts.sweeps)
                                                                 for r, _, _, _ in jobs),
                           "algorithmic_terms_per_step": algo_terms_total, "evaluated_terms_per_step": actual_terms,
                           "reference_cost_evals_per_step": ref_evals,
                           "reference_terms_per_step": ref_rows5 * 5},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in head_kt.items() if v[1]},
            "fused_points": head_pts,
            "setup_s": setup_s,
            "kernels": ("one-candidate init" if opts.flags & 1 else
                        "row-step init" if opts.flags & 128 else "table-sweep init"),
            "schedule": {"tile": f"{opts.tile_w}x{opts.tile_h}" if opts.tile_w else "8x8 (library default)",
                         "threads_per_pixel": max(opts.threads_per_pixel, 1), "flags": opts.flags,
                         "persistent_queue": bool(opts.flags & 2), "cuda_graph": bool(opts.flags & 4),
                         "autotuned_tiles": bool(opts.flags & 8), "tune_table": ctx.tune_table()},
        }
        print(json.dumps(line), flush=True)
    if net is not None:
        net.close()
    ds.close()
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
