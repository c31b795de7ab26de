"""B200-native dense multi-view stereo: census patch-match stereo and
geometric-consistency fusion behind the C ABI of include/rcmvs.h.

The compute path lives in librcmvs.so (CUDA, sm_100a); this package holds its
Python host mirror (rustcolmap_b200.mvs), data types, the build script and
the synthetic scene generator.
"""
from .types import Cam, DepthMap, MvsOptions, MvsStats, SparseModel, ViewData  # noqa: F401

__version__ = "0.1.0"
