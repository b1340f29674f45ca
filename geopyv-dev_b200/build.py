"""Build recipe for the in-tree native libraries (sm_100a only).

    python geopyv-dev_b200/build.py [--force]

Produces, next to the Python package that loads them:
    gpv/libgpv_b200.so   -- the C-ABI library (include/gpv.h): CUDA kernels + host API
    gpv/libgpvsynth.so   -- seeded synthetic speckle generator (inputs for tests/benchmarks)
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "gpv")
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _gomp_dir() -> str:
    hits = sorted(glob.glob("/usr/lib/gcc/x86_64-linux-gnu/*/libgomp.spec"))
    return os.path.dirname(hits[-1]) if hits else ""


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    deps = srcs + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "gpv.h")]
    target = os.path.join(OUT, "libgpv_b200.so")
    if not force and not _stale(target, deps):
        return target
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O3",
           "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-o", target, *srcs, "-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return target


def build_synth(force: bool = False) -> str:
    src = os.path.join(CSRC, "synth.c")
    target = os.path.join(OUT, "libgpvsynth.so")
    if not force and not _stale(target, [src]):
        return target
    cc = os.environ.get("CC", "gcc")
    cmd = [cc, "-O3", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-o", target, src, "-lm"]
    g = _gomp_dir()
    if g:
        cmd.insert(1, "-B" + g + "/")
    subprocess.run(cmd, check=True)
    return target


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_synth(force)
    build_cuda(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
