"""Builds the in-tree CUDA library ``imageprocessingflex_b200/lib/libipfcuda.so``.

Every ``csrc/*.cu`` file is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with ``nvcc`` and linked into one
shared library exposing the C ABI of ``include/ipfc.h``.  Objects are cached
under ``lib/obj/`` and rebuilt when a source or header is newer.  Compiles run
in parallel (one process per file).

Usage: ``python -m imageprocessingflex_b200.build [--force] [-v]``
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIBNAME = "libipfcuda.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fvisibility=hidden",
    "-I", os.path.join(ROOT, "include"),
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libipfcuda.so")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, verbose: bool) -> None:
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
    if os.path.basename(src).startswith(("sep_fast_", "batch_", "sep_tcol")):
        cmd.insert(1, "--split-compile=4")  # many kernels or tile functions per file: compile them in parallel
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles what is stale and links the library; returns its path."""
    os.makedirs(OBJDIR, exist_ok=True)
    # the heavy instantiation files first, so the pool's tail is short
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")),
                  key=lambda p: (not os.path.basename(p).startswith(("batch_heavy", "sep_fast_")), p))
    hdrs = _headers()
    jobs = []
    objs = []
    for src in srcs:
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda j: _compile(j[0], j[1], verbose), jobs))
    if force or jobs or _stale(LIBPATH, objs):
        tmp = LIBPATH + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(tmp, LIBPATH)
    return LIBPATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
