"""Builds the in-tree shared libraries with nvcc for sm_100a.

librcmvs.so   — the stereo + fusion path behind include/rcmvs.h
librcscene.so — the synthetic scene renderer behind include/rcscene.h

Both build with --fmad=false and IEEE divide / square root: the stereo and
fusion kernels reproduce the reference's f32/f64 results bit for bit, and the
renderer gives identical images on host and device.  Objects are rebuilt
only when a source or header is newer than the library.

    python -m rustcolmap_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(CSRC, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-Xptxas", "-warn-spills",
]

LIBS = {
    "librcmvs.so": ["capi.cu", "census.cu", "stereo.cu", "fuse.cu", "noalloc.cu", "learned.cu", "learned_api.cu",
                   "schedule.cu", "depthvis.cu", "resize.cu", "sift.cu", "match.cu"],
    "librcscene.so": ["scene.cu"],
}
LINK = {"librcmvs.so": ["-lz"]}  # zlib: the grey PNG writer
HEADERS = [os.path.join(CSRC, "rcmvs_internal.cuh"), os.path.join(CSRC, "ctx_internal.cuh"),
           os.path.join(CSRC, "learned.cuh"), os.path.join(ROOT, "include", "rcmvs.h"),
           os.path.join(ROOT, "include", "rcscene.h")]


def _newer(src_paths, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in src_paths)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    out = []
    for lib, srcs in LIBS.items():
        target = os.path.join(HERE, lib)
        objs = []
        for s in srcs:
            src = os.path.join(CSRC, s)
            obj = os.path.join(BUILD, s.replace(".cu", ".o"))
            if force or _newer([src] + HEADERS, obj):
                cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
                if verbose:
                    print(" ".join(cmd))
                subprocess.run(cmd, check=True)
            objs.append(obj)
        if force or _newer(objs, target):
            cmd = [NVCC] + ARCH + ["-shared", "-o", target] + objs + LINK.get(lib, [])
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        out.append(target)
    return out


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv, verbose=True):
        print("built", p)
