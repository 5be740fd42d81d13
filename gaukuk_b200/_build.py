"""Builds the native parts of gaukuk_b200 in-tree.

* ``lib/libgk_cuda.so`` -- the CUDA kernels and the C ABI of
  include/gaukuk_cuda.h, compiled for sm_100a only.  The parity unit is
  compiled with ``-fmad=false`` (no FMA contraction), the fast unit without.
* ``lib/libgaukuk_host.so`` and ``bin/gaukuk_<setup>.sim`` -- the C++ host
  layer that keeps the reference's classes (see gaukuk_b200/src), built by
  ``build_host()``.

Rebuilds only what is older than its sources.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")
OBJ = os.path.join(PKG, "lib", "obj")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-I" + INCLUDE, "-I" + CSRC]

CUDA_LIB = os.path.join(LIB, "libgk_cuda.so")


def _newer(target: str, deps: List[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: List[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)


def build_cuda(verbose: bool = False, force: bool = False) -> str:
    """Compile the CUDA units and link libgk_cuda.so; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    units = {
        "gk_kernels_parity.cu": ["-fmad=false"],
        "gk_kernels_fast.cu": [],
        "gk_api.cu": [],
    }
    extra = sorted(os.path.basename(p) for p in glob.glob(os.path.join(CSRC, "*.cu")))
    for name in extra:
        units.setdefault(name, [])
    objs = []
    for name, flags in units.items():
        src = os.path.join(CSRC, name)
        obj = os.path.join(OBJ, name.replace(".cu", ".o"))
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            _run([NVCC] + NVCC_FLAGS + flags + ["-c", src, "-o", obj], verbose)
    if force or _newer(CUDA_LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", CUDA_LIB] + objs, verbose)
    return CUDA_LIB


def build_all(verbose: bool = False, force: bool = False) -> None:
    build_cuda(verbose=verbose, force=force)
    try:
        from . import _build_host
    except ImportError:
        return
    _build_host.build_host(verbose=verbose, force=force)


def clean() -> None:
    for d in (LIB, BIN):
        if os.path.isdir(d):
            shutil.rmtree(d)
