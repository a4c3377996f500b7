"""Builds libpincflow_poisson.so (the C-ABI solver library) for sm_100a.

Usage: python pincflow.jl_b200/build.py [--force] [--verbose] [--checked]

The library is written in-tree to pincflow.jl_b200/lib/ so that it travels
with the repository snapshot.  --checked builds the bounds-checked variant
libpincflow_poisson_checked.so (-DPCF_BOUNDS_CHECK: every instrumented
global index is checked against its array's extent; pcf_bounds_check_status
reports the first failure).  Each .cu file is compiled separately (in
parallel) and linked with nvcc; a file is rebuilt when it or any header is
newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OBJDIR = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpincflow_poisson.so")
OBJDIR_CHECKED = os.path.join(HERE, "_build_checked")
LIB_CHECKED = os.path.join(LIBDIR, "libpincflow_poisson_checked.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers())


def _compile(src: str, verbose: bool, objdir: str = OBJDIR, extra=()) -> str:
    obj = os.path.join(objdir, os.path.basename(src).replace(".cu", ".o"))
    cmd = [NVCC] + ARCH + FLAGS + list(extra) + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    objdir, lib = (OBJDIR_CHECKED, LIB_CHECKED) if checked else (OBJDIR, LIB)
    extra = ["-DPCF_BOUNDS_CHECK"] if checked else []
    os.makedirs(objdir, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    obj_of = lambda s: os.path.join(objdir, os.path.basename(s).replace(".cu", ".o"))  # noqa: E731
    todo = [s for s in srcs if force or _stale(s, obj_of(s))]
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(todo)))) as ex:
        list(ex.map(lambda s: _compile(s, verbose, objdir, extra), todo))
    objs = [obj_of(s) for s in srcs]
    if force or todo or not os.path.exists(lib):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--checked", action="store_true")
    args = ap.parse_args()
    print(build(args.force, args.verbose, args.checked))
