"""Build libpsi_b200.so (CUDA, sm_100a) and the PSI CPython extension in-tree.

    python pypsi_b200/build.py [--force] [-v]

Objects go to pypsi_b200/_build/; the two shared libraries land next to this
file so they travel with the source tree.  FMA contraction is disabled in every
translation unit except clip_mixed.cu and bfs.cu (the mixed walks): the FP64
path repeats the reference's double-precision operation order.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libpsi_b200.so")
EXT = os.path.join(HERE, "PSI" + sysconfig.get_config_var("EXT_SUFFIX"))

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_UNITS = {  # unit -> extra flags
    "clip_fp64.cu": ["--fmad=false"],
    "clip_mixed.cu": [],
    "tess.cu": ["--fmad=false"],
    "pipeline.cu": ["--fmad=false"],
    "annihilation_host.cu": ["--fmad=false"],
    "query_host.cu": ["--fmad=false"],
    "noalloc.cu": ["--fmad=false"],
    "bfs.cu": [],
    "bfs_fp64.cu": ["--fmad=false"],
    "annihilation.cu": ["--fmad=false"],
    "probe.cu": [],  # the FMA issue-rate probe (explicit fma(), so contraction does not matter)
    "loaders.cpp": [],  # host code only: the snapshot readers
}
HEADERS = ["psib_device.cuh", "psib_clip.cuh", "psib_kernels.h", "psib_accum.cuh", "psib_adjoint.cuh",
           "psib_bfs.cuh", "pipeline_host.h"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "psi_b200.h")]
    objs, jobs = [], []
    for unit, extra in CUDA_UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, os.path.splitext(unit)[0] + ".o")
        objs.append(obj)
        if force or _newer(obj, [src, __file__] + hdrs):
            jobs.append([NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I",
                         CSRC, *extra, "-c", src, "-o", obj])
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    if force or _newer(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-o", LIB, *objs], verbose)
    msrc = os.path.join(CSRC, "psi_module.c")
    if force or _newer(EXT, [msrc, LIB, os.path.join(INCLUDE, "psi_b200.h")]):
        import numpy as np
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-Wall", "-Wno-missing-field-initializers",
              "-I", sysconfig.get_paths()["include"], "-I", np.get_include(), "-I", INCLUDE, msrc,
              "-L", HERE, "-lpsi_b200", "-Wl,-rpath,$ORIGIN", "-o", EXT], verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
