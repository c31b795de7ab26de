import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) GPU; runs the librcmvs kernels")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU here")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


GOLDEN = os.path.join(ROOT, "tests", "golden", "tiny_corner.npz")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def golden_views(g):
    """ViewData list rebuilt from the golden fixture."""
    from rustcolmap_b200.types import Cam, ViewData
    views = []
    i = 0
    while f"gray{i}" in g:
        gray = g[f"gray{i}"]
        h, w = gray.shape
        cam = g[f"cam{i}"]
        views.append(ViewData(f"v{i}", i, w, h, Cam(*cam), g[f"R{i}"], g[f"t{i}"], gray,
                              np.repeat(gray[:, :, None], 3, axis=2)))
        i += 1
    return views


@pytest.fixture(scope="session")
def corner_scene():
    from rustcolmap_b200 import scene
    return scene.corner_room(seed=0)


@pytest.fixture(scope="session")
def c1_opts():
    from rustcolmap_b200 import MvsOptions
    # "6 red-black iterations" = sweeps 6 (12 passes), 64 hypotheses, K = 4
    return MvsOptions(max_dim=4096, num_sources=4, sweeps=6, num_hyp=64)
