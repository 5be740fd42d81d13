"""ctypes front end to the checkers (TEST INFRASTRUCTURE ONLY).

* ``OracleSim`` drives the plain-C restatement in ``oracle/_build/libgk_oracle.so``.
* ``run_reference`` runs the reference itself (``oracle/_ref/ref_strict`` or
  ``ref_fast``, built from the reference sources by oracle/Makefile) on any
  initial state and returns the final state and the full-precision dt log.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module; the product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import tempfile
from typing import List, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgk_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class GkoParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("ng", ctypes.c_int),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
        ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
        ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
        ("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
        ("integrator", ctypes.c_int), ("rc_order", ctypes.c_int),
        ("bc", ctypes.c_int * 6), ("grav", ctypes.c_double * 3),
        ("dfloor", ctypes.c_double), ("pfloor", ctypes.c_double),
        ("stepmax", ctypes.c_int),
    ]


# callbacks of gko_advance_split: halo(user, state), reduce(user, local) -> max
HALO_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double))
MAX_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_void_p, ctypes.c_double)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle lib)")
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.gko_create.restype = ctypes.c_void_p
        L.gko_create.argtypes = [ctypes.POINTER(GkoParams)]
        L.gko_destroy.argtypes = [ctypes.c_void_p]
        L.gko_state_size.restype = ctypes.c_longlong
        L.gko_state_size.argtypes = [ctypes.c_void_p]
        L.gko_set_cons.argtypes = [ctypes.c_void_p, dp]
        L.gko_get_cons.argtypes = [ctypes.c_void_p, dp]
        L.gko_update_bd.argtypes = [ctypes.c_void_p]
        L.gko_cmax.restype = ctypes.c_double
        L.gko_cmax.argtypes = [ctypes.c_void_p]
        L.gko_advance.restype = ctypes.c_int
        L.gko_advance.argtypes = [ctypes.c_void_p, ctypes.c_double, dp, ctypes.c_int]
        for name in ("gko_time", "gko_dt"):
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [ctypes.c_void_p]
        for name in ("gko_step", "gko_is_continue"):
            getattr(L, name).restype = ctypes.c_int
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.gko_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.gko_hllc_batch.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_double, dp]
        L.gko_vanleer_batch.argtypes = [ctypes.c_int, dp, dp, dp]
        L.gko_cons_to_prim_batch.argtypes = [ctypes.c_int, dp, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, dp]
        L.gko_set_spacing.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double]
        L.gko_advance_split.restype = ctypes.c_int
        L.gko_advance_split.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, HALO_FN,
                                        MAX_FN, ctypes.c_void_p, dp, ctypes.c_int]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def to_gko_params(p) -> GkoParams:
    g = GkoParams()
    for f in ("nx", "ny", "nz", "ng", "integrator", "rc_order", "stepmax"):
        setattr(g, f, int(getattr(p, f)))
    for f in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "gamma", "cfl", "dfloor", "pfloor"):
        setattr(g, f, float(getattr(p, f)))
    for i in range(6):
        g.bc[i] = int(p.bc[i])
    for i in range(3):
        g.grav[i] = float(p.grav[i])
    return g


class OracleSim:
    """The C restatement of Sim (sim.cpp) on one reference-layout state."""

    def __init__(self, params, cons: Optional[np.ndarray] = None):
        self.params = params
        self._gp = to_gko_params(params)
        self.h = lib().gko_create(ctypes.byref(self._gp))
        if not self.h:
            raise ValueError("oracle rejected the parameters")
        if cons is not None:
            self.set_cons(cons)

    def __del__(self):
        if getattr(self, "h", None):
            lib().gko_destroy(self.h)
            self.h = None

    def set_cons(self, cons):
        c = np.ascontiguousarray(cons, dtype=np.float64)
        assert c.size == lib().gko_state_size(self.h)
        lib().gko_set_cons(self.h, _dp(c))

    def get_cons(self) -> np.ndarray:
        out = np.empty(self.params.shape, dtype=np.float64)
        lib().gko_get_cons(self.h, _dp(out))
        return out

    def update_bd(self):
        lib().gko_update_bd(self.h)

    def cmax(self) -> float:
        return lib().gko_cmax(self.h)

    def advance(self, dtoutput: float, cap: int = 1 << 20) -> List[float]:
        buf = np.empty(cap, dtype=np.float64)
        n = lib().gko_advance(self.h, float(dtoutput), _dp(buf), cap)
        return buf[:min(n, cap)].tolist()

    def run(self, tmax: float, dtoutput: float) -> List[float]:
        """The output-cadence loop of main.cpp:44-52 (without the writes)."""
        dts: List[float] = []
        t = self.time
        while abs(tmax - t) > 1e-12 and self.is_continue:
            dtoutput = min(dtoutput, tmax - t)
            dts += self.advance(dtoutput)
            t = self.time
        return dts

    @property
    def time(self) -> float:
        return lib().gko_time(self.h)

    @property
    def step(self) -> int:
        return lib().gko_step(self.h)

    @property
    def is_continue(self) -> bool:
        return bool(lib().gko_is_continue(self.h))


def hllc_batch(wl: np.ndarray, wr: np.ndarray, direction: int, gamma: float) -> np.ndarray:
    wl = np.ascontiguousarray(wl, dtype=np.float64)
    wr = np.ascontiguousarray(wr, dtype=np.float64)
    n = wl.shape[1]
    out = np.empty((5, n), dtype=np.float64)
    lib().gko_hllc_batch(n, _dp(wl), _dp(wr), int(direction), float(gamma), _dp(out))
    return out


def vanleer_batch(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.empty_like(a)
    lib().gko_vanleer_batch(a.size, _dp(a), _dp(b), _dp(out))
    return out


def reference_available(flavour: str = "strict") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"ref_{flavour}"))


_STEP_RE = re.compile(r"^step = (\d+), t = (\S+), dt = (\S+)$")


def run_reference(params, cons: np.ndarray, tmax: Optional[float] = None,
                  dtoutput: Optional[float] = None, stepmax: Optional[int] = None,
                  flavour: str = "strict", threads: Optional[int] = None,
                  timeout: float = 600.0) -> Tuple[np.ndarray, List[float], dict]:
    """Run the reference build on ``cons``; returns (final cons, dt log, stats).

    The dt log is parsed from the reference's own per-step lines
    (sim.cpp:100-103), printed with 17 significant digits by the driver."""
    import json
    exe = os.path.join(REF_DIR, f"ref_{flavour}")
    if not os.path.exists(exe):
        raise RuntimeError(f"reference build missing: {exe}")
    tmax = params.tmax if tmax is None else tmax
    dtoutput = params.dtoutput if dtoutput is None else dtoutput
    stepmax = params.stepmax if stepmax is None else stepmax
    c = np.ascontiguousarray(cons, dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        inf = os.path.join(td, "run.in")
        icf = os.path.join(td, "ic.bin")
        outf = os.path.join(td, "out.bin")
        import dataclasses
        p2 = dataclasses.replace(params, tmax=tmax, dtoutput=dtoutput, stepmax=stepmax)
        with open(inf, "w") as f:
            f.write(p2.to_in_text())
        c.tofile(icf)
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run([exe, "-i", inf, "--ic", icf, "--out", outf], cwd=td,
                           capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-2000:]}")
        out = np.fromfile(outf, dtype=np.float64).reshape(params.shape)
        dts = []
        for line in r.stdout.splitlines():
            m = _STEP_RE.match(line.strip())
            if m:
                dts.append(float(m.group(3)))
        stats = json.loads(r.stderr.strip().splitlines()[-1])
    return out, dts, stats
