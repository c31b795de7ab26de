#!/usr/bin/env python
"""Benchmark of the dense-MVS hot path on B200 (one JSON line on rank 0).

Workload (default, --config c5): the full-scale synthetic scene — 100 views at
1920x1080 of a room + 60 boxes + 10 spheres, f = 1.15 x 1920, K = 10 support
views, 64 plane-sweep hypotheses, 6 sweeps (12 Jacobi passes), fusion with
>= 3 consistent views, 1% relative depth agreement and a 1 px reprojection
gate.  One step = census + rays, patch-match stereo for all 100 views, and
geometric-consistency fusion with voxel dedup (the PLY vertex records are
packed on the device).

value  depth maps/s with inputs resident in HBM (rcmvs_scene_* calls), timed
       with CUDA events on the library's stream, max over ranks.
e2e    the same metric through rcmvs_run_mvs with pinned host buffers:
       host->device copy of every view's grey + colour image, device->host
       read of the fused cloud, inside the timed region.

--impl reference times the reference algorithm's CPU implementation (the
oracle port; the Rust reference cannot be built here) on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c5|c2|c1]
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


def configs():
    from rustcolmap_b200 import MvsOptions
    return {
        "c5": dict(desc="100 views 1920x1080, room + 60 boxes + 10 spheres, f=1.15*1920, K=10, 64 hyps, "
                        "6 sweeps (12 passes); fusion min_consistent=3, depth_diff=0.01, reprojection <= 1 px",
                   scene=dict(n_views=100, sizes=((1920, 1080),), f_rel=1.15, n_boxes=60, n_spheres=10),
                   opts=MvsOptions(max_dim=1920, num_sources=10, sweeps=6, num_hyp=64, min_consistent=3,
                                   depth_diff=0.01, reproj_px=1.0)),
        "c2": dict(desc="64 views 960x720, room + 20 boxes, f=1.1*960, K=8, 64 hyps, 6 sweeps (12 passes)",
                   scene=dict(n_views=64, sizes=((960, 720),), f_rel=1.1, n_boxes=20, n_spheres=0),
                   opts=MvsOptions(max_dim=960, num_sources=8, sweeps=6, num_hyp=64)),
        "c1": dict(desc="corner room, 8 views 384x288, f=440, K=4, 64 hyps, 6 sweeps (12 passes)",
                   scene=None, opts=MvsOptions(max_dim=384, num_sources=4, sweeps=6, num_hyp=64)),
    }


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


def cpu_baseline(sc, opts, jobs, rows, threads=0):
    """Times the oracle's estimate_depth on a band of `rows` rows of the first
    job's reference view (a bounded sample of one view).  Returns (depth
    maps/s, seconds, sample description, threads)."""
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
            f"{v.w}x{v.h} view, K={len(srcs)}, {opts.num_hyp} hyps, {2 * opts.sweeps} passes; "
            f"{frac:.4f} of a depth map per sample, stereo only")
    return frac / dt, dt, desc, nt


def run_reference(args, cfg):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    from rustcolmap_b200 import mvs
    oracle.lib()
    sc = make_scene(cfg, seed=5, device=-1 if not _has_gpu() else 0)
    opts = cfg["opts"]
    srcs, zr, fus = mvs.plan(sc.sparse, sc.views, opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(sc.views)) if srcs[i]]
    rows = args.ref_rows
    for _ in range(args.warmup):
        cpu_baseline(sc, opts, jobs, rows)
    times, rate, desc, nt = [], 0.0, "", 0
    for _ in range(args.steps):
        r, dt, desc, nt = cpu_baseline(sc, opts, jobs, rows)
        times.append(dt)
    frac = rows / sc.views[jobs[0][0]].h
    rate = frac * len(times) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "depth maps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": args.config + ": " + cfg["desc"]},
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


METRIC = "1080p depth maps/s at K=10 (plain GPU patch-match + fusion; learned init not in this number)"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=["c5", "c2", "c1"])
    ap.add_argument("--cpu-rows", type=int, default=24, help="rows of the CPU-baseline band")
    ap.add_argument("--ref-rows", type=int, default=12, help="rows per step of the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--views", type=int, default=0, help="override the number of views (profiling runs)")
    ap.add_argument("--no-count", action="store_true", help="skip the work-counting rerun")
    ap.add_argument("--one-candidate", action="store_true",
                    help="use the one-candidate-at-a-time stereo kernels (comparison)")
    args = ap.parse_args()
    assert args.warmup >= 3 or os.environ.get("RCMVS_BENCH_ALLOW_SHORT"), "warm-up must be >= 3 steps"
    cfg = configs()[args.config]
    if args.views and cfg["scene"] is not None:
        cfg["scene"] = dict(cfg["scene"], n_views=args.views)
        cfg["desc"] += f" [{args.views} views]"
    if args.impl == "reference":
        run_reference(args, cfg)
        return

    import torch

    from rustcolmap_b200 import mvs, scene
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    opts = cfg["opts"]
    if args.one_candidate:
        opts.flags |= 1
    t_setup = time.perf_counter()
    sc = make_scene(cfg, seed=5 + 1000 * rank, device=local)
    srcs, zr, fus = mvs.plan(sc.sparse, sc.views, opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(sc.views)) if srcs[i]]
    n_maps = len(jobs)
    ctx = mvs.Context(local)
    ds = mvs.DeviceScene(sc.views, ctx)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    setup_s = time.perf_counter() - t_setup

    def step():
        ds.prepare()
        ds.estimate(jobs, opts)
        return ds.fuse(fus, sc.sparse.xyz, opts)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    barrier(ws)
    clk = ClockSampler(local)
    clk.start()
    ctx.timing(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(ws)
    e0.record(stream)
    n_points = 0
    for _ in range(args.steps):
        n_points = step()
    e1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    barrier(ws)
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    ktimes = {k: ctx.kernel_time(k) for k in ("census_rays", "stereo_init", "stereo_pass", "stereo_gate",
                                              "fuse_candidates", "fuse_reduce")}
    ctx.timing(False)
    ms_max = max_over_ranks(ms, ws, local)
    total_maps = sum_over_ranks(n_maps * args.steps, ws, local)
    value = total_maps / (ms_max / 1e3)

    # work counters (untimed rerun with counting on): actual cost evaluations and rows
    evals, rows5 = 0, 0
    if not args.no_count:
        os.environ["RCMVS_COUNT"] = "1"
        cctx = mvs.Context(local)
        del os.environ["RCMVS_COUNT"]
        cds = mvs.DeviceScene(sc.views, cctx)
        cds.estimate(jobs, opts)
        evals, rows5 = cctx.last_work()
        cds.close()
        cctx.close()

    # end to end through the reference-facing call with pinned host buffers
    e2e = None
    if not args.no_e2e:
        pv = pinned_views(sc.views)
        mvs.run_mvs(pv, sc.sparse, opts, ctx=ctx)  # warm
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            st, xyz, rgb = mvs.run_mvs(pv, sc.sparse, opts, ctx=ctx)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        barrier(ws)
        dt = max_over_ranks(dt, ws, local)
        h2d = int(sum(v.gray.nbytes + v.rgb.nbytes for v in pv))
        e2e = {"value": sum_over_ranks(n_maps * args.steps, ws, local) / dt, "unit": "depth maps/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(xyz.nbytes + rgb.nbytes),
               "ms_per_step": 1e3 * dt / args.steps}

    # ground-truth error of this step's depth maps
    accs, comps = [], []
    for (ref, _, _, _) in jobs[:: max(1, len(jobs) // 20)]:
        m = scene.gt_metrics(ds.depth(ref).depth, sc.gt_depth[ref])
        accs.append(m["accuracy"])
        comps.append(m["completeness"])

    # roofline of the dominant kernel (the Jacobi pass)
    npx = sum(sc.views[r].w * sc.views[r].h for r, _, _, _ in jobs)
    src_px = sum(sc.views[s].w * sc.views[s].h for _, ss, _, _ in jobs for s in ss)
    K = max(len(s) for _, s, _, _ in jobs)
    pass_ms, pass_n = ktimes["stereo_pass"]
    pass_avg_s = pass_ms / max(pass_n, 1) / 1e3
    bytes_per_launch = npx * (20 + 20 + 8 + 8) + src_px * 8
    achieved_gbs = bytes_per_launch / pass_avg_s / 1e9
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    terms_alg_per_pass = npx * 7 * 25 * sum(len(s) for _, s, _, _ in jobs) / len(jobs)
    algo_terms_total = sum(sc.views[r].w * sc.views[r].h * 25 * len(s) * (opts.num_hyp + 7 * 2 * opts.sweeps)
                           for r, s, _, _ in jobs)
    actual_terms = rows5 * 5
    step_s = ms_max / 1e3 / args.steps
    stereo_ms = sum(ktimes[k][0] for k in ("stereo_init", "stereo_pass", "stereo_gate")) / args.steps
    fp32_ops_per_term = 40
    achieved_tops = actual_terms * fp32_ops_per_term / (stereo_ms / 1e3) / 1e12 if actual_terms else None

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and ws == 1:
        rate, dt, desc, nt = cpu_baseline(sc, opts, jobs, args.cpu_rows)
        cpu = {"value": rate, "unit": "depth maps/s", "cores": nt, "kind": "port", "sample": desc,
               "seconds": dt}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "depth maps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config + ": " + cfg["desc"], "views_per_step": n_maps,
                       "parallelism": f"views batched on 1 GPU; {ws} rank(s), one independent scene each",
                       "l2": "inputs larger than L2 (census 8 B/px, rays 8 B/px, planes 40 B/px over all views)"},
            "roofline": {"bound": "hbm", "kernel": "stereo_pass", "achieved": achieved_gbs, "peak": hbm_peak,
                         "unit": "GB/s", "frac": achieved_gbs / hbm_peak, "traffic": None,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650",
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "avg_launch_ms": pass_avg_s * 1e3,
                         "note": "issue-bound kernel: see compute_roofline"},
            "compute_roofline": {"bound": "fp32_issue", "achieved": achieved_tops, "peak": FP32_NOMINAL_TOPS,
                                 "unit": "Top/s",
                                 "frac": achieved_tops / FP32_NOMINAL_TOPS if achieved_tops else None,
                                 "ops_per_term": fp32_ops_per_term,
                                 "peak_source": "nominal 148 SM x 128 FP32 lanes x 1.965 GHz"},
            "gpu_launches": args.steps * (1 + 1 + 2 * opts.sweeps + 1 + 5),
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gcost_evals_per_s": evals * args.steps / (ms_max / 1e3) / 1e9,
            "work": {"cost_evals_per_step": evals, "window_rows_per_step": rows5,
                     "algorithmic_cost_evals_per_step": sum(sc.views[r].w * sc.views[r].h *
                                                           (opts.num_hyp + 14 * opts.sweeps) for r, _, _, _ in jobs),
                     "algorithmic_terms_per_step": algo_terms_total, "evaluated_terms_per_step": actual_terms},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in ktimes.items()},
            "fused_points": n_points,
            "gt": {"accuracy_median": statistics.median(accs), "completeness_median": statistics.median(comps),
                   "tol": "1% relative inverse depth", "views_sampled": len(accs)},
            "setup_s": setup_s,
            "kernels": "one-candidate" if opts.flags & 1 else "row-step",
        }
        print(json.dumps(line), flush=True)
    ds.close()
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
