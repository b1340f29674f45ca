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


OBJ = os.path.join(HERE, "_build")  # per-source objects (git-ignored)
FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    """Each source compiles to its own object (recompiled when it, a local
    header or include/gpv.h is newer), then one link; sources compile in
    parallel."""
    from concurrent.futures import ThreadPoolExecutor
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "gpv.h")]
    target = os.path.join(OUT, "libgpv_b200.so")
    os.makedirs(OBJ, exist_ok=True)
    objs, jobs = [], []
    for src in srcs:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers]):
            cmd = [NVCC, *FLAGS, "-I" + os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for r in ex.map(lambda c: subprocess.run(c, capture_output=not verbose, text=True), jobs):
            if r.returncode != 0:
                sys.stderr.write((r.stdout or "") + (r.stderr or ""))
                raise subprocess.CalledProcessError(r.returncode, r.args)
    if jobs or force or _stale(target, objs):
        subprocess.run([NVCC, *ARCH, "-shared", "-o", target, *objs, "-lcudart"], check=True)
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
