"""Builds libm2s.so in place from csrc/*.cu with nvcc for sm_100a.

    python -m mesh_to_sdf_b200.build [--force] [--verbose]

The library links the CUDA runtime statically, so it loads next to any
PyTorch build without a libcudart version clash.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libm2s.so")
FAST_LIB = os.path.join(HERE, "libm2s_fast.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
         "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(ROOT, "include", "m2s.h"))
    return hdrs


def lib_path(fast: bool = False) -> str:
    return FAST_LIB if fast else LIB


def up_to_date(fast: bool = False) -> bool:
    lib = lib_path(fast)
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in sources() + _deps() + [__file__])


def build(force: bool = False, verbose: bool = False, fast: bool = False) -> str:
    """The strict build (libm2s.so: every distance operation rounds like the
    reference) or, with fast=True, the fast build (libm2s_fast.so: compiled
    with M2S_FAST_MATH, multiply-adds fused in the closest-point and distance
    arithmetic only)."""
    lib = lib_path(fast)
    if not force and up_to_date(fast):
        return lib
    bdir = os.path.join(BUILD, "fast") if fast else BUILD
    os.makedirs(bdir, exist_ok=True)
    cc = nvcc()
    defs = ["-DM2S_FAST_MATH"] if fast else []

    def compile_one(src):
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmd = [cc, *ARCH, *FLAGS, *defs, "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, sources()))
    if verbose:
        for _, err in results:
            sys.stderr.write(err)
    objs = [o for o, _ in results]
    tmp = lib + ".tmp"
    r = subprocess.run([cc, *ARCH, "-shared", "-o", tmp, *objs], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    fast = "--fast" in sys.argv
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, fast=fast))
