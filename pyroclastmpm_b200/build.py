"""Build the native parts in-tree: libpmpm_b200.so (sm_100a kernels + C ABI)
and the MPM2D / MPM3D Python extension modules.  nvcc cross-compiles for
sm_100a without a GPU."""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libpmpm_b200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_lib(verbose=False, force=False):
    srcs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    deps = srcs + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [os.path.join(INCLUDE, "pmpm.h")]
    if force or _stale(LIB, deps):
        _run(["nvcc", *NVCC_FLAGS, f"-I{INCLUDE}", "-o", LIB, *srcs], verbose)
    return LIB


def build_modules(verbose=False, force=False):
    """pybind11 modules MPM2D / MPM3D (the reference module names), one per
    dimension as the reference builds them (-DDIM)."""
    import pybind11

    src = os.path.join(HERE, "cpp", "bindings.cpp")
    if not os.path.exists(src):
        return []
    deps = [src] + sorted(glob.glob(os.path.join(HERE, "cpp", "*.hpp"))) + [os.path.join(INCLUDE, "pmpm.h"), LIB]
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = []
    for dim in (2, 3):
        target = os.path.join(HERE, f"MPM{dim}D{ext}")
        if force or _stale(target, deps):
            _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-Wall", f"-DDIM={dim}",
                  f"-I{INCLUDE}", f"-I{os.path.join(HERE, 'cpp')}", f"-I{pybind11.get_include()}",
                  f"-I{sysconfig.get_paths()['include']}", src, "-o", target,
                  f"-L{HERE}", "-l:libpmpm_b200.so", "-Wl,-rpath,$ORIGIN"], verbose)
        out.append(target)
    return out


def build_all(verbose=False, force=False):
    build_lib(verbose, force)
    build_modules(verbose, force)


if __name__ == "__main__":
    build_all(verbose=True, force="--force" in sys.argv)
