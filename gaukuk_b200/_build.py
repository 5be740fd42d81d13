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


CHECKED_LIB = os.path.join(LIB, "checked", "libgk_cuda.so")


def build_cuda(verbose: bool = False, force: bool = False, checked: bool = False) -> str:
    """Compile the CUDA units and link libgk_cuda.so; returns its path.
    checked=True builds the bounds-checked variant (GK_CHECKED: coordinates
    checked and clamped, counters read by gk_checked_report) into
    lib/checked/, for tests; the product path loads it only with
    GK_CHECKED=1."""
    obj_dir = os.path.join(OBJ, "checked") if checked else OBJ
    lib_path = CHECKED_LIB if checked else CUDA_LIB
    os.makedirs(obj_dir, exist_ok=True)
    os.makedirs(os.path.dirname(lib_path), exist_ok=True)
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
    objs, cmds = [], []
    extra_flags = ["-DGK_CHECKED=1"] if checked else []
    for name, flags in units.items():
        src = os.path.join(CSRC, name)
        obj = os.path.join(obj_dir, name.replace(".cu", ".o"))
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            cmds.append([NVCC] + NVCC_FLAGS + flags + extra_flags + ["-c", src, "-o", obj])
    # the units compile independently: one nvcc per unit at a time
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, c, verbose) for c in cmds]:
            f.result()
    if force or _newer(lib_path, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", lib_path] + objs, verbose)
    return lib_path


def build_all(verbose: bool = False, force: bool = False) -> None:
    build_cuda(verbose=verbose, force=force)
    build_cuda(verbose=verbose, force=force, checked=True)
    try:
        from . import _build_host
    except ImportError:
        return
    _build_host.build_host(verbose=verbose, force=force)


def clean() -> None:
    for d in (LIB, BIN):
        if os.path.isdir(d):
            shutil.rmtree(d)
