"""Builds the C++ host layer (gaukuk_b200/src) and one driver per problem hook.

* ``lib/libgaukuk_host.a`` -- Config, Grid/Domain, EquationOfState,
  Boundary, SourceTerm, Sim (whose Advance calls libgk_cuda.so), WriteData.
* ``bin/gaukuk_<name>.sim`` -- main.cpp + the host library + one problem hook
  ``src/setup/setup_<name>.cpp``, linked against lib/libgk_cuda.so: the
  reference's ``gaukuk.sim -i file.in`` with the time loop on the GPU.

The host code is compiled without FMA contraction or fast-math, so a hook
computes the same initial state bits as the reference built with strict IEEE
flags.  ``build_hook(path)`` builds a driver for any hook file written for
the reference -- the hook's own ``#include "../sim.hpp"`` resolves to this
layer's headers (``-I-`` stops the compiler from looking next to the hook).
Where the reference's sources are given (``GK_REFERENCE_SRC``, else the
checkout the oracle recipe last built from, recorded in oracle/_ref/SOURCE),
its own setup files that run on the device path are built as well,
unchanged, as ``bin/gaukuk_ref_<name>.sim``.  With neither, they are
skipped.
"""
from __future__ import annotations

import glob
import os
from typing import List, Optional

from ._build import BIN, CUDA_LIB, INCLUDE, LIB, OBJ, PKG, _newer, _run, build_cuda

SRC = os.path.join(PKG, "src")
SETUP = os.path.join(SRC, "setup")
HOST_LIB = os.path.join(LIB, "libgaukuk_host.a")
CXX = "g++"
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
            "-Wno-unused-variable", "-I" + INCLUDE, "-I" + SRC]
HOST_SRCS = ["sim.cpp", "utils/read_config.cpp", "utils/write_sim.cpp", "eos/adiabatic.cpp",
             "boundary/boundary.cpp", "source_term/source.cpp"]


def _headers() -> List[str]:
    return glob.glob(os.path.join(SRC, "**", "*.hpp"), recursive=True) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def build_host_lib(verbose: bool = False, force: bool = False) -> str:
    odir = os.path.join(OBJ, "host")
    os.makedirs(odir, exist_ok=True)
    objs = []
    for rel in HOST_SRCS + ["main.cpp"]:
        src = os.path.join(SRC, rel)
        obj = os.path.join(odir, rel.replace("/", "_").replace(".cpp", ".o"))
        if force or _newer(obj, [src] + _headers()):
            _run([CXX] + CXXFLAGS + ["-c", src, "-o", obj], verbose)
        if rel != "main.cpp":
            objs.append(obj)
    if force or _newer(HOST_LIB, objs):
        if os.path.exists(HOST_LIB):
            os.remove(HOST_LIB)
        _run(["ar", "rcs", HOST_LIB] + objs, verbose)
    return HOST_LIB


def build_hook(hook_src: str, name: Optional[str] = None, verbose: bool = False,
               force: bool = False, out_dir: str = BIN) -> str:
    """Links bin/gaukuk_<name>.sim from main.cpp, the host library and a hook."""
    build_cuda(verbose=verbose)
    build_host_lib(verbose=verbose)
    name = name or os.path.basename(hook_src)[len("setup_"):-len(".cpp")]
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, f"gaukuk_{name}.sim")
    main_obj = os.path.join(OBJ, "host", "main.o")
    if force or _newer(exe, [hook_src, main_obj, HOST_LIB, CUDA_LIB]):
        # -I- : quote includes of the hook are looked up in -I directories
        # only, so "../sim.hpp" from a hook file anywhere resolves to src/.
        cmd = [CXX] + CXXFLAGS + ["-I-", "-I" + SETUP, "-o", exe, hook_src, main_obj, HOST_LIB,
                                  "-L" + LIB, "-lgk_cuda", "-Wl,-rpath," + LIB]
        _run(cmd, verbose)
    return exe


def reference_src() -> str:
    """The reference checkout: GK_REFERENCE_SRC, else the path the oracle
    recipe recorded when it built from it, else '' (none given)."""
    env = os.environ.get("GK_REFERENCE_SRC", "")
    if env:
        return env
    rec = os.path.join(os.path.dirname(PKG), "oracle", "_ref", "SOURCE")
    if os.path.exists(rec):
        with open(rec) as f:
            return f.read().strip()
    return ""


REFERENCE_SRC = reference_src()
REFERENCE_HOOKS = ("blast", "disk", "disk_planet", "example", "kh", "rt", "shock_tube", "solid_body",
                   "wave_test")


def build_host(verbose: bool = False, force: bool = False) -> None:
    build_host_lib(verbose=verbose, force=force)
    for hook in sorted(glob.glob(os.path.join(SETUP, "setup_*.cpp"))):
        build_hook(hook, verbose=verbose, force=force)
    ref = reference_src()
    for name in REFERENCE_HOOKS:
        src = os.path.join(ref, "src", "setup", f"setup_{name}.cpp")
        if ref and os.path.exists(src):
            build_hook(src, name="ref_" + name, verbose=verbose, force=force)


SANITIZE = ["-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
            "-fno-sanitize-recover=undefined"]


def build_sanitized(hooks: List[str], out_dir: str, verbose: bool = False) -> List[str]:
    """The host layer under AddressSanitizer and UndefinedBehaviorSanitizer:
    compiles its sources once into out_dir and links one driver per hook
    (``<out_dir>/gaukuk_<name>.asan``) against lib/libgk_cuda.so.  Strict IEEE
    flags are kept, so the drivers write the same frames as the plain ones."""
    build_cuda(verbose=verbose)
    os.makedirs(out_dir, exist_ok=True)
    flags = [f for f in CXXFLAGS if f != "-O2"] + SANITIZE
    objs = []
    for rel in HOST_SRCS + ["main.cpp"]:
        obj = os.path.join(out_dir, rel.replace("/", "_").replace(".cpp", ".o"))
        _run([CXX] + flags + ["-c", os.path.join(SRC, rel), "-o", obj], verbose)
        objs.append(obj)
    exes = []
    for hook in hooks:
        name = os.path.basename(hook)[len("setup_"):-len(".cpp")]
        exe = os.path.join(out_dir, f"gaukuk_{name}.asan")
        _run([CXX] + flags + ["-I-", "-I" + SETUP, "-o", exe, hook] + objs +
             ["-L" + LIB, "-lgk_cuda", "-Wl,-rpath," + LIB], verbose)
        exes.append(exe)
    return exes
