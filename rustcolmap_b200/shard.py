"""One scene on several GPUs: one process per GPU (torch.distributed),
reference views sharded across ranks for stereo and for fusion.

The reference runs `estimate_depth` for every view in a rayon `par_iter`
(mvs/src/lib.rs:345-370) and then `fuse_depth_maps` over all of them
(mvs/src/lib.rs:426).  Stereo for one reference view reads only its own and
its sources' census (read-only), so views shard across ranks with no
exchange.  Each rank recomputes the census of all views itself (17 bytes per
pixel of HBM traffic, a few ms for 100 1080p views) instead of receiving it:
that is cheaper than the collective and needs no synchronisation.

Fusion checks each reference pixel against the depth maps of the views in
its fusion order, so one all-gather of the depth maps follows stereo.  Then
each rank runs the consistency check (fuse.rs:96-167) for the pixels of its
own reference views, the candidates of all ranks are all-gathered and
concatenated in view order, which is the order the reference accumulates
them in, and every rank runs the voxel dedup (fuse.rs:176-214) on the same
list.

Every rank takes the same collective steps in the same order.  The result
is bit-identical to the single-GPU `mvs.run_mvs` (each view's stereo, each
pixel's check and the dedup are the same computations; only where they run
changes).

Two data planes: `run_mvs_sharded_device` keeps the scene resident on each
rank's GPU and moves depth maps and candidates device to device through the
collectives (the NCCL path); `run_mvs_sharded` moves them through host
arrays, with pluggable stereo/fusion back ends.
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


def all_gather_candidates(xyz, rgb, per_view, group=None, device="cpu"):
    """All-gather fusion candidates and concatenate them in view order.

    xyz (n, 3) f64, rgb (n, 3) u8: this rank's candidates in view-then-pixel
    order; per_view (n_views,): this rank's count per view (0 for views it
    did not check; every view is checked by at most one rank).  Returns
    (xyz, rgb) of all ranks' candidates, view by view in ascending order,
    the same on every rank.  One all_gather of the counts, one of the
    candidates packed as 4 f64 each (x, y, z, r | g << 8 | b << 16, exact),
    padded to the largest rank's count."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8).reshape(-1, 3)
    counts = np.ascontiguousarray(per_view, dtype=np.int64)
    if counts.sum() != len(xyz) or len(rgb) != len(xyz):
        raise ValueError("per-view counts do not add up to the candidates")
    nv = len(counts)
    head = np.concatenate([[len(xyz)], counts]).astype(np.int64)
    heads = [torch.empty(nv + 1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(heads, torch.from_numpy(head).to(device), group=group)
    heads = [h.cpu().numpy() for h in heads]
    n_max = max(1, max(int(h[0]) for h in heads))
    buf = np.zeros((n_max, 4), np.float64)
    buf[:len(xyz), :3] = xyz
    c = rgb.astype(np.int64)
    buf[:len(xyz), 3] = c[:, 0] | (c[:, 1] << 8) | (c[:, 2] << 16)
    parts = [torch.empty((n_max, 4), dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(parts, torch.from_numpy(buf).to(device), group=group)
    parts = [p.cpu().numpy() for p in parts]
    pieces, cursor = [], [0] * world
    for v in range(nv):
        for r in range(world):
            k = int(heads[r][1 + v])
            if k:
                pieces.append(parts[r][cursor[r]:cursor[r] + k])
                cursor[r] += k
    allc = np.concatenate(pieces) if pieces else np.zeros((0, 4), np.float64)
    packed = allc[:, 3].astype(np.int64)
    out_rgb = np.stack([packed & 255, (packed >> 8) & 255, (packed >> 16) & 255], axis=1).astype(np.uint8)
    return np.ascontiguousarray(allc[:, :3]), out_rgb


def run_mvs_sharded(views, sparse, opts, group=None, ctx=None, stereo=None, candidates=None, reduce=None,
                    device="cpu"):
    """`run_mvs` with this scene's reference views spread over the ranks of
    `group`, for stereo and for fusion.  Returns (fused xyz (n,3) f64, rgb
    (n,3) u8, depth maps per view or None) on every rank.

    stereo(jobs) -> {view: depth (h, w)} runs this rank's jobs (default: the
    library on this rank's GPU through a DeviceScene);
    candidates(depth_maps, fusion_order, ref_views) -> (xyz, rgb, per_view)
    checks this rank's reference pixels (default: `mvs.fuse_candidates`);
    reduce(xyz, rgb) -> (xyz, rgb) dedups all candidates (default:
    `mvs.fuse_reduce`).  They are parameters so that the host logic can be
    exercised with other back ends."""
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
    if candidates is None:
        def candidates(dm, order, refs):
            return mvs.fuse_candidates(views, dm, order, refs, opts, ctx)
    if reduce is None:
        def reduce(cx, cc):
            return mvs.fuse_reduce(cx, cc, sparse.xyz, opts, ctx)
    cx, cc, per_view = candidates(depth, fus, sorted(r for r, _, _, _ in mine))
    ax, ac = all_gather_candidates(cx, cc, per_view, group=group, device=device)
    xyz, rgb = reduce(ax, ac)
    return xyz, rgb, depth


# ------------------------------------------------- device data plane
class SceneOps:
    """The scene operations the device data plane needs, on this rank's GPU
    through the library (one DeviceScene kept for the whole run).  Tensors
    passed in are CUDA tensors of this rank's device; the library works on
    its own stream, so `sync()` separates its writes from the collectives'
    reads, and the caller synchronises the collectives' stream before the
    library reads what they wrote."""

    def __init__(self, views, opts, ctx, net=None, **learned_kw):
        self.views, self.opts = views, opts
        self.net, self.learned_kw = net, learned_kw
        self.ds = mvs.DeviceScene(views, ctx)

    def stereo(self, jobs):
        """Census of every view (sources may be other ranks' views), then
        this rank's jobs: plain stereo, or seeded by the proposal network
        when one was given."""
        self.ds.prepare()
        if not jobs:
            return
        if self.net is None:
            self.ds.estimate(jobs, self.opts)
        else:
            from . import learned
            learned.estimate_learned(self.ds, jobs, self.opts, self.net, **self.learned_kw)

    def depth_into(self, v, t):
        self.ds.depth_to_device(v, t.data_ptr())

    def set_depth(self, v, t):
        self.ds.set_depth(v, t.data_ptr())

    def candidates(self, fusion_order, refs):
        return self.ds.fuse_candidates_device(fusion_order, refs, self.opts)

    def candidates_into(self, xyz, rgb):
        self.ds.candidates_to_device(xyz.data_ptr(), rgb.data_ptr())

    def reduce(self, xyz, rgb, n, sparse_xyz):
        self.ds.fuse_reduce_device(xyz.data_ptr(), rgb.data_ptr(), n, sparse_xyz, self.opts)
        return self.ds.points()

    def depth_host(self, v):
        return self.ds.depth(v).depth

    def sync(self):
        self.ds.ctx.synchronize()

    def close(self):
        self.ds.close()


def _stream_sync(device):
    import torch
    if torch.device(device).type == "cuda":
        torch.cuda.current_stream(device).synchronize()


def gather_maps_device(ops, shapes, owners, group=None, device="cuda"):
    """All-gather of the per-view depth maps between devices: each rank's
    maps go from its scene into one send tensor (device to device), one
    all_gather moves every rank's tensor, and each received map goes into
    this rank's scene (device to device).  No host copy of a map."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    per_rank = [sorted(v for v, o in owners.items() if o == r) for r in range(world)]
    sizes = [sum(int(np.prod(shapes[v])) for v in views) for views in per_rank]
    n = max(max(sizes), 1)
    send = torch.zeros(n, dtype=torch.float32, device=device)
    o = 0
    for v in per_rank[rank]:
        k = int(np.prod(shapes[v]))
        ops.depth_into(v, send[o:o + k])
        o += k
    ops.sync()
    parts = [torch.empty(n, dtype=torch.float32, device=device) for _ in range(world)]
    dist.all_gather(parts, send, group=group)
    _stream_sync(device)
    for r in range(world):
        if r == rank:
            continue
        o = 0
        for v in per_rank[r]:
            k = int(np.prod(shapes[v]))
            ops.set_depth(v, parts[r][o:o + k])
            o += k
    ops.sync()
    return parts  # kept alive until the library's copies have run


def gather_candidates_device(ops, n_mine, per_view, group=None, device="cuda"):
    """All-gather of the fusion candidates between devices, concatenated in
    view order (the reference's accumulation order): one all_gather of the
    per-view counts (small, read on the host to cut the pieces), one of the
    positions (f64) and one of the colours (u8), each padded to the largest
    rank's count.  Returns (xyz (N, 3) f64, rgb (N, 3) u8) tensors on
    `device`, the same on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    nv = len(per_view)
    head = torch.tensor([int(n_mine)] + [int(c) for c in per_view], dtype=torch.int64, device=device)
    heads = [torch.empty(nv + 1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(heads, head, group=group)
    heads = [h.cpu().numpy() for h in heads]
    n_max = max(1, max(int(h[0]) for h in heads))
    sx = torch.zeros((n_max, 3), dtype=torch.float64, device=device)
    sc = torch.zeros((n_max, 3), dtype=torch.uint8, device=device)
    if n_mine:
        ops.candidates_into(sx, sc)
    ops.sync()
    px = [torch.empty((n_max, 3), dtype=torch.float64, device=device) for _ in range(world)]
    pc = [torch.empty((n_max, 3), dtype=torch.uint8, device=device) for _ in range(world)]
    dist.all_gather(px, sx, group=group)
    dist.all_gather(pc, sc, group=group)
    pieces_x, pieces_c, cursor = [], [], [0] * world
    for v in range(nv):
        for r in range(world):
            k = int(heads[r][1 + v])
            if k:
                pieces_x.append(px[r][cursor[r]:cursor[r] + k])
                pieces_c.append(pc[r][cursor[r]:cursor[r] + k])
                cursor[r] += k
    if not pieces_x:
        return (torch.zeros((0, 3), dtype=torch.float64, device=device),
                torch.zeros((0, 3), dtype=torch.uint8, device=device))
    ax, ac = torch.cat(pieces_x).contiguous(), torch.cat(pieces_c).contiguous()
    _stream_sync(device)
    return ax, ac


def run_mvs_sharded_device(views, sparse, opts, group=None, ctx=None, device=None, ops=None, planner=None,
                           return_depth=False):
    """run_mvs_sharded with the data plane on the devices: the scene stays
    resident on each rank's GPU from census to fusion, depth maps and
    candidates move device to device through the collectives (NCCL over
    NVLink with a `nccl` group), and the only host copy is the fused cloud
    at the end.  Returns (xyz (n, 3) f64, rgb (n, 3) u8, depth maps or
    None).  ops: the scene operations (default SceneOps, the library on this
    rank's GPU; the CPU tests pass the oracle behind the same methods);
    planner: the host glue (default the library's rcmvs_plan)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    planner = planner or mvs.plan
    srcs, zr, fus = planner(sparse, views, opts)
    jobs = [(i, srcs[i], zr[i, 0], zr[i, 1]) for i in range(len(views)) if srcs[i]]
    parts = assign_views(job_costs(jobs, views), world)
    owners = {jobs[j][0]: r for r in range(world) for j in parts[r]}
    mine = [jobs[j] for j in parts[rank]]
    own = ops is None
    if own:
        ctx = ctx or mvs.default_context()
        ops = SceneOps(views, opts, ctx)
        device = device or f"cuda:{ctx.device}"
    device = device or "cpu"
    try:
        ops.stereo(mine)
        shapes = {r: (views[r].h, views[r].w) for r, _, _, _ in jobs}
        keep = gather_maps_device(ops, shapes, owners, group=group, device=device)
        n_mine, per_view = ops.candidates(fus, sorted(r for r, _, _, _ in mine))
        ax, ac = gather_candidates_device(ops, n_mine, per_view, group=group, device=device)
        xyz, rgb = ops.reduce(ax, ac, len(ax), sparse.xyz)
        depth = [ops.depth_host(i) if i in shapes else None for i in range(len(views))] if return_depth else None
        del keep
    finally:
        if own:
            ops.close()
    return xyz, rgb, depth


# ------------------------------------------------------------ SfM front end
def _gather_items(local, n_items, group=None, device="cpu"):
    """All-gather variable-size float64 vectors keyed 0..n_items-1, each
    produced on exactly one rank: local = {item: 1-D array}.  Returns
    {item: array} for every item, the same on every rank.  One all_gather of
    the per-rank sizes and item lengths, one of the data padded to the
    largest rank's size."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    lens = np.full(n_items, -1, np.int64)
    for k, v in local.items():
        lens[k] = len(v)
    flat = np.concatenate([np.asarray(local[k], np.float64).ravel() for k in sorted(local)]) if local \
        else np.zeros(0, np.float64)
    head = np.concatenate([[len(flat)], lens]).astype(np.int64)
    heads = [torch.empty(n_items + 1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(heads, torch.from_numpy(head).to(device), group=group)
    heads = [h.cpu().numpy() for h in heads]
    n_max = max(1, max(int(h[0]) for h in heads))
    buf = np.zeros(n_max, np.float64)
    buf[:len(flat)] = flat
    parts = [torch.empty(n_max, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(parts, torch.from_numpy(buf).to(device), group=group)
    out = {}
    for r in range(world):
        data = parts[r].cpu().numpy()
        o = 0
        for k in range(n_items):
            ln = int(heads[r][1 + k])
            if ln >= 0:
                out[k] = data[o:o + ln].copy()
                o += ln
    return out


def _pack_frame(f):
    n = len(f.pts)
    return np.concatenate([[f.width, f.height, n, f.n_raw], f.pts.ravel(), f.desc.ravel().astype(np.float64),
                           f.colors.ravel().astype(np.float64)])


def _unpack_frame(v, name):
    from .sift import DESC_LEN, SiftFrame
    w, h, n, n_raw = (int(x) for x in v[:4])
    o = 4
    pts = v[o:o + 2 * n].reshape(n, 2).copy()
    o += 2 * n
    desc = v[o:o + DESC_LEN * n].astype(np.float32).reshape(n, DESC_LEN)
    o += DESC_LEN * n
    col = v[o:o + 3 * n].astype(np.uint8).reshape(n, 3)
    return SiftFrame(name, w, h, pts, desc, col, n_raw)


def extract_and_match_sharded(images, names=None, opts=None, ratio=0.75, sequential=False, group=None, ctx=None,
                              extract=None, match=None, device="cpu"):
    """sift.extract_and_match with images and pairs spread over the ranks of
    `group`: each rank extracts the SIFT features of its share of the images
    (longest-processing-time order on pixel counts), the frames are
    all-gathered, each rank matches its share of the job pairs (by na * nb),
    and the matches are all-gathered.  Returns (frames, pairs, matches) on
    every rank, equal to the single-process result (the same computations,
    spread differently; descriptors travel as exact f64).

    extract(image, name) -> SiftFrame and match(descs, pairs) -> [(a, b)]
    default to the library on this rank's GPU; they are parameters so that
    the host logic can run with other back ends."""
    import torch.distributed as dist
    from . import sift
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = len(images)
    if n < 2:
        raise sift.RcmvsError(-1, "need at least 2 images")
    names = names or [""] * n
    if extract is None:
        def extract(im, nm):
            return sift.extract_sift(im, nm, opts, ctx)
    if match is None:
        def match(descs, prs):
            return sift.match_pairs(descs, prs, ratio, ctx)
    img_parts = assign_views([int(np.asarray(im).shape[0]) * int(np.asarray(im).shape[1]) for im in images], world)
    local = {i: _pack_frame(extract(images[i], names[i])) for i in img_parts[rank]}
    packed = _gather_items(local, n, group, device)
    frames = [_unpack_frame(packed[i], names[i]) for i in range(n)]
    pairs = sift.job_pairs(n, sequential)
    pair_parts = assign_views([max(len(frames[i].pts) * len(frames[j].pts), 1) for i, j in pairs], world)
    mine = pair_parts[rank]
    got = match([f.desc for f in frames], [pairs[p] for p in mine]) if mine else []
    local_m = {p: np.concatenate([a, b]).astype(np.float64) for p, (a, b) in zip(mine, got)}
    allm = _gather_items(local_m, len(pairs), group, device)
    matches = []
    for p in range(len(pairs)):
        v = allm[p].astype(np.uint32)
        k = len(v) // 2
        matches.append((v[:k], v[k:]))
    return frames, pairs, matches
