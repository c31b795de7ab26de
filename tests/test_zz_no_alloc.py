"""rcmvs_estimate_depth_noalloc: estimate_depth for callers that may not
allocate device memory.

Such a caller owns its GPU memory through another allocator (here torch's
caching allocator stands in for it) or runs in a loop that cannot take the
device-wide synchronisation of cudaMalloc/cudaFree.  It hands the entry point
device buffers it allocated itself; the entry point keeps its intermediates
in one fixed __device__ array.  The test checks two calls in a row against
the allocating entry point (bit for bit, the tolerance of every stereo parity
test here) and that the second call leaves the device's free memory as it
was.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from rustcolmap_b200 import MvsOptions, _abi, _lib, mvs

pytestmark = pytest.mark.gpu


def _device_views(views, torch, dev):
    grays = [torch.from_numpy(np.ascontiguousarray(v.gray)).to(dev) for v in views]
    va = _abi.view_array(views)
    for i, g in enumerate(grays):
        va[i].gray = g.data_ptr()
        va[i].rgb = None
    return va, grays


def test_noalloc_matches_allocating_entry_point_on_two_calls(corner_scene):
    import torch
    views = corner_scene.views
    opts = MvsOptions(max_dim=4096, num_sources=4, sweeps=6, num_hyp=64)
    srcs, zr, _ = mvs.plan(corner_scene.sparse, views, opts)
    refs = [0, 5]
    ctx = mvs.Context(0)
    expected = [mvs.estimate_depth(views, r, srcs[r], zr[r, 0], zr[r, 1], opts, ctx) for r in refs]
    ctx.close()

    dev = torch.device("cuda:0")
    va, keep = _device_views(views, torch, dev)
    h, w = views[0].h, views[0].w
    outs = [(torch.full((h, w), -7.0, dtype=torch.float32, device=dev),
             torch.full((h, w), -7.0, dtype=torch.float32, device=dev)) for _ in refs]
    o = opts.to_c()
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = _lib.mvs()
    torch.cuda.synchronize()
    free = []
    for r, (d, c) in zip(refs, outs):
        s = np.ascontiguousarray(srcs[r], dtype=np.int32)
        free.append(torch.cuda.mem_get_info(dev)[0])
        rc = L.rcmvs_estimate_depth_noalloc(va, len(views), r, s.ctypes.data, len(s), float(zr[r, 0]),
                                            float(zr[r, 1]), C.byref(o), d.data_ptr(), c.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info(dev)[0])
    for (d, c), e in zip(outs, expected):
        assert np.array_equal(d.cpu().numpy().view(np.uint32), e.depth.view(np.uint32))
        assert np.array_equal(c.cpu().numpy().view(np.uint32), e.cost.view(np.uint32))
    assert free[2] == free[1], "the second call changed the device's free memory"


def test_noalloc_rejects_sizes_beyond_its_limits(corner_scene):
    import torch
    from rustcolmap_b200.types import Cam, ViewData
    dev = torch.device("cuda:0")
    big = torch.zeros((481, 640), dtype=torch.uint8, device=dev)  # one row over 640 x 480
    v = ViewData("big", 0, 640, 481, Cam(600.0, 320.0, 240.0), np.eye(3), np.zeros(3),
                 np.zeros((481, 640), np.uint8))
    va = _abi.view_array([v, v])
    va[0].gray = va[1].gray = big.data_ptr()
    o = MvsOptions(max_dim=4096).to_c()
    d = torch.empty((481, 640), dtype=torch.float32, device=dev)
    one = np.array([1], np.int32)
    L = _lib.mvs()
    rc = L.rcmvs_estimate_depth_noalloc(va, 2, 0, one.ctypes.data, 1, 1.0, 5.0, C.byref(o), d.data_ptr(),
                                        d.data_ptr(), None)
    assert rc == _abi.RCMVS_E_LIMIT
    va2, keep = _device_views(corner_scene.views, torch, dev)
    five = np.array([1, 2, 3, 4, 5], np.int32)  # one source over the limit of 4
    rc = L.rcmvs_estimate_depth_noalloc(va2, len(corner_scene.views), 0, five.ctypes.data, 5, 1.0, 5.0,
                                        C.byref(o), d.data_ptr(), d.data_ptr(), None)
    assert rc == _abi.RCMVS_E_LIMIT
    assert _abi.RCMVS_E_LIMIT == -4
