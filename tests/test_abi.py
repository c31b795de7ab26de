"""The C-ABI libraries load and export everything include/*.h declares; host
entry points that need no GPU behave like the reference (no compute calls on
a GPU here)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, has_gpu
from oracle import oracle
from rustcolmap_b200 import MvsOptions, _abi, _lib, mvs


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:rcmvs|rcscene)_\w+)\s*\(", src)))


def _exported(so):
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


@pytest.mark.parametrize("header,so", [("rcmvs.h", "librcmvs.so"), ("rcscene.h", "librcscene.so")])
def test_library_exports_every_declared_symbol(header, so):
    path = os.path.join(ROOT, "rustcolmap_b200", so)
    C.CDLL(path)  # loads without a GPU
    decl = _declared(header)
    assert decl, "no declarations parsed"
    missing = [d for d in decl if d not in _exported(path)]
    assert not missing, missing


def test_python_signature_table_covers_header():
    assert set(_lib.exported_symbols()) == set(_declared("rcmvs.h"))


def test_abi_struct_layouts_match_c(tmp_path):
    prog = tmp_path / "layout.c"
    prog.write_text(r"""
#include <stdio.h>
#include <stddef.h>
#include "rcmvs.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(rcmvs_options), sizeof(rcmvs_view), sizeof(rcmvs_job),
         sizeof(rcmvs_depth_out), sizeof(rcmvs_sparse), sizeof(rcmvs_points), sizeof(rcmvs_stats));
  printf("%zu %zu %zu %zu\n", offsetof(rcmvs_options, depth_diff), offsetof(rcmvs_options, reproj_px),
         offsetof(rcmvs_view, gray), offsetof(rcmvs_job, zmin));
  return 0; }
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    offs = [int(x) for x in lines[1].split()]
    assert sizes == [C.sizeof(t) for t in (_abi.Options, _abi.View, _abi.Job, _abi.DepthOut, _abi.Sparse,
                                           _abi.Points, _abi.Stats)]
    assert offs == [_abi.Options.depth_diff.offset, _abi.Options.reproj_px.offset, _abi.View.gray.offset,
                    _abi.Job.zmin.offset]


def test_options_default_mirrors_mvsoptions_default():
    o = _abi.Options()
    _lib.mvs().rcmvs_options_default(C.byref(o))
    ref = MvsOptions().to_c()
    for name, _ in _abi.Options._fields_:
        assert getattr(o, name) == getattr(ref, name), name
    # lib.rs:56-70
    assert (o.max_dim, o.num_sources, o.sweeps, o.num_hyp, o.min_consistent) == (900, 3, 4, 48, 2)
    assert o.depth_diff == 0.03 and abs(o.cost_thr - 0.38) < 1e-7 and o.voxel_rel == 0.0015


def test_pass_count():
    """2 * max(sweeps, 1) passes (stereo.rs:271) unless the passes extension
    is set; none with RCMVS_FLAG_INIT_ONLY."""
    from rustcolmap_b200.types import FLAG_INIT_ONLY
    n = lambda **kw: _lib.mvs().rcmvs_pass_count(C.byref(MvsOptions(**kw).to_c()))
    assert n(sweeps=6) == 12 and n(sweeps=0) == 2 and n(sweeps=1) == 2 and n(sweeps=3) == 6
    assert n(sweeps=3, passes=5) == 5 and n(sweeps=6, passes=1) == 1
    assert n(sweeps=3, passes=5, flags=FLAG_INIT_ONLY) == 0 and n(sweeps=6, flags=FLAG_INIT_ONLY) == 0


def test_write_ply_matches_oracle(tmp_path):
    rng = np.random.default_rng(0)
    xyz = rng.normal(size=(257, 3))
    rgb = rng.integers(0, 256, (257, 3), dtype=np.uint8)
    a, b = str(tmp_path / "a.ply"), str(tmp_path / "b.ply")
    mvs.write_ply_binary(a, xyz, rgb)
    oracle.write_ply_binary(b, xyz, rgb)
    assert open(a, "rb").read() == open(b, "rb").read()
    mvs.write_ply_binary(a, xyz[:0], rgb[:0])
    assert open(a, "rb").read().endswith(b"element vertex 0\nproperty float x\nproperty float y\nproperty float z\n"
                                         b"property uchar red\nproperty uchar green\nproperty uchar blue\n"
                                         b"end_header\n")


def test_plan_matches_oracle(corner_scene, c1_opts):
    a = mvs.plan(corner_scene.sparse, corner_scene.views, c1_opts)
    b = oracle.plan(corner_scene.sparse, corner_scene.views, c1_opts)
    assert a[0] == b[0] and a[2] == b[2]
    assert np.array_equal(a[1], b[1])
    assert all(len(s) == 4 for s in a[0])


@pytest.mark.parametrize("n_views,per_view,k", [(24, 120, 8), (100, 300, 10)])
def test_plan_matches_oracle_orbit(n_views, per_view, k):
    """The library's plan (threaded co-visibility, depth percentiles by
    selection) against the oracle's sequential one; the second case has the
    C5 workload's view count and sparse density."""
    from rustcolmap_b200 import scene
    sc = scene.orbit_room(seed=3, n_views=n_views, sizes=((96, 72),), n_boxes=8, per_view_sparse=per_view)
    o = MvsOptions(num_sources=k)
    a = mvs.plan(sc.sparse, sc.views, o)
    b = oracle.plan(sc.sparse, sc.views, o)
    assert a[0] == b[0] and a[2] == b[2] and np.array_equal(a[1], b[1])


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_context_without_gpu_fails_loudly():
    with pytest.raises(_lib.RcmvsError):
        mvs.Context(0)


def test_package_has_no_cpu_fallback():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "rustcolmap_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                assert "oracle" not in open(os.path.join(dirpath, f)).read().replace("the oracle", ""), f


@pytest.mark.parametrize("n,cap", [(5000, 700), (5000, 0), (1, 0), (2, 1), (37, 5)])
def test_dense_outputs_match_oracle(tmp_path, n, cap):
    """dense_web.json (mvs/src/lib.rs:434-485) against the oracle's plain
    Python restatement on a fixed-order cloud with outliers; dense.ply
    against the PLY writer; mvs_stats.json's format."""
    rng = np.random.default_rng(n + cap)
    xyz = rng.normal(size=(n, 3)) * [2.0, 1.0, 0.5] + [10.0, -3.0, 4.0]
    if n > 10:
        xyz[:: max(n // 20, 1)] *= 40.0  # far outliers, dropped from the web copy
    rgb = rng.integers(0, 256, (n, 3), dtype=np.uint8)
    stats = mvs.MvsStats(views=12, views_with_depth=11, dense_points=n, per_view_valid=[], elapsed_s=3.25,
                         stereo_s=1.04, fuse_s=0.96, fusion_candidates=0)
    mvs.write_dense_outputs(str(tmp_path), xyz, rgb, stats, web_cap=cap)
    assert open(tmp_path / "dense_web.json").read() == oracle.web_json(xyz, rgb, cap or 400_000)
    oracle.write_ply_binary(str(tmp_path / "o.ply"), xyz, rgb)
    assert open(tmp_path / "dense.ply", "rb").read() == open(tmp_path / "o.ply", "rb").read()
    assert open(tmp_path / "mvs_stats.json").read() == (
        '{"views": 12, "views_with_depth": 11, "dense_points": %d, "stereo_s": 1.0, "fuse_s": 1.0, '
        '"elapsed_s": %.1f}' % (n, np.float32(3.25)))


def test_dense_outputs_of_an_empty_cloud(tmp_path):
    mvs.write_dense_outputs(str(tmp_path), np.zeros((0, 3)), np.zeros((0, 3), np.uint8))
    assert (tmp_path / "dense.ply").exists() and not (tmp_path / "dense_web.json").exists()


def test_surface_distance_of_the_synthetic_scenes():
    """The fused-cloud ground truth: points sampled from the rendered depth
    maps lie on the analytic surfaces, and points moved off a wall, a box
    face and a sphere by a known amount are that far away."""
    from rustcolmap_b200 import scene
    sc = scene.orbit_room(seed=4, n_views=3, sizes=((64, 48),), n_boxes=4, n_spheres=2, per_view_sparse=60)
    d = scene.surface_distance(sc.sparse.xyz, sc.prims)
    assert d.max() < 1e-4, d.max()
    walls = scene.surface_distance(np.array([[0.0, 0.0, 2.0], [5.5, 0.3, 1.0], [0.1, -0.2, -0.25]]), sc.prims[:5])
    np.testing.assert_allclose(walls, [2.0, 0.5, 0.25], atol=1e-12)
    box = scene.SyntheticScene([], [], None, None, "t", 0, [scene._box((0, 0, 0), (1, 2, 3), np.random.default_rng(0))])
    sph = scene._sphere((5.0, 0.0, 0.0), 0.5, np.random.default_rng(0))
    got = scene.surface_distance(np.array([[0.5, 1.0, 1.0], [2.0, 1.0, 1.5], [0.5, 1.0, 3.25]]), box.prims)
    np.testing.assert_allclose(got, [0.5, 1.0, 0.25], atol=1e-12)
    np.testing.assert_allclose(scene.surface_distance(np.array([[5.0, 0.0, 1.0], [5.0, 0.1, 0.0]]), [sph]),
                               [0.5, 0.4], atol=1e-12)
