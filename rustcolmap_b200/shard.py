"""One scene on several GPUs: one process per GPU (torch.distributed),
reference views sharded across ranks, depth maps all-gathered for fusion.

The reference runs `estimate_depth` for every view in a rayon `par_iter`
(mvs/src/lib.rs:345-370) and then `fuse_depth_maps` over all of them
(mvs/src/lib.rs:426).  Stereo for one reference view reads only its own and
its sources' census (read-only), so views shard across ranks with no
exchange; fusion needs every view's depth map, so one all-gather precedes
it.  Each rank recomputes the census of all views itself (17 bytes per pixel
of HBM traffic, a few ms for 100 1080p views) instead of receiving it: that
is cheaper than the collective and needs no synchronisation.

Every rank takes the same collective steps in the same order.  The result
is bit-identical to the single-GPU `mvs.run_mvs` (each view's stereo and the
fusion are the same computations; only where they run changes).
"""
import numpy as np

from . import mvs


def job_costs(jobs, views):
    """Work estimate per job: reference pixels x support views."""
    return [views[r].w * views[r].h * max(len(s), 1) for r, s, _, _ in jobs]


def assign_views(costs, world):
    """Longest-processing-time assignment of jobs to `world` ranks: jobs in
    decreasing cost (ties: lower index first), each to the least-loaded rank
    (ties: lower rank).  Returns one ascending list of job indices per rank;
    the same on every rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


def all_gather_maps(local, shapes, owners, group=None, device="cpu"):
    """All-gather per-view float32 maps.

    local:  {view: (h, w) array} computed on this rank
    shapes: {view: (h, w)} of every view in the job list (same on all ranks)
    owners: {view: rank} (same on all ranks)
    Returns {view: (h, w) float32 array} for every view in `shapes`.  Each
    rank sends its maps concatenated in ascending view order, padded to the
    largest rank's length (one all_gather of equal-size tensors); `device`
    is where the tensors live ("cuda" for NCCL, "cpu" for gloo)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    per_rank = [sorted(v for v, o in owners.items() if o == r) for r in range(world)]
    sizes = [sum(int(np.prod(shapes[v])) for v in views) for views in per_rank]
    n = max(max(sizes), 1)
    buf = np.zeros(n, np.float32)
    o = 0
    for v in per_rank[rank]:
        a = np.ascontiguousarray(local[v], dtype=np.float32).ravel()
        if a.size != int(np.prod(shapes[v])):
            raise ValueError(f"view {v}: map has {a.size} values, expected {shapes[v]}")
        buf[o:o + a.size] = a
        o += a.size
    mine = torch.from_numpy(buf).to(device)
    parts = [torch.empty(n, dtype=torch.float32, device=device) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = {}
    for r in range(world):
        flat = parts[r].cpu().numpy()
        o = 0
        for v in per_rank[r]:
            k = int(np.prod(shapes[v]))
            out[v] = flat[o:o + k].reshape(shapes[v]).copy()
            o += k
    return out


def run_mvs_sharded(views, sparse, opts, group=None, ctx=None, stereo=None, fuse=None, device="cpu"):
    """`run_mvs` with this scene's reference views spread over the ranks of
    `group`.  Returns (fused xyz (n,3) f64, rgb (n,3) u8, depth maps per
    view or None) on every rank.

    stereo(jobs) -> {view: depth (h, w)} runs this rank's jobs (default: the
    library on this rank's GPU through a DeviceScene); fuse(depth_maps,
    fusion_order) -> (xyz, rgb) fuses (default: `mvs.fuse_depth_maps`).
    Both are parameters so that the host logic can be exercised with other
    back ends."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    srcs, zr, fus = mvs.plan(sparse, views, opts)  # host glue: deterministic on every rank
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(views)) if srcs[i]]
    parts = assign_views(job_costs(jobs, views), world)
    owners = {jobs[j][0]: r for r in range(world) for j in parts[r]}
    mine = [jobs[j] for j in parts[rank]]
    if stereo is None:
        def stereo(js):
            if not js:
                return {}
            ds = mvs.DeviceScene(views, ctx)
            try:
                ds.prepare()
                ds.estimate(js, opts)
                return {r: ds.depth(r).depth for r, _, _, _ in js}
            finally:
                ds.close()
    local = stereo(mine)
    shapes = {r: (views[r].h, views[r].w) for r, _, _, _ in jobs}
    maps = all_gather_maps(local, shapes, owners, group=group, device=device)
    depth = [maps.get(i) for i in range(len(views))]
    if fuse is None:
        def fuse(dm, order):
            return mvs.fuse_depth_maps(views, dm, order, sparse.xyz, opts, ctx)
    xyz, rgb = fuse(depth, fus)
    return xyz, rgb, depth
