"""Python front end of the device finite-volume update.

``Sim`` mirrors the reference's ``Gaukuk::Sim`` (src/sim.hpp:23-58): it holds
the state of one problem, ``advance(dtoutput)`` is ``Sim::Advance``
(sim.cpp:69-117), ``get_time/get_dt/get_step`` and ``is_continue`` are the
reference accessors, and ``run(tmax, dtoutput)`` is the output-cadence loop of
main.cpp:44-52.  States cross the boundary in the reference's TArray layout,
``cons[n][k][j][i]``.  All work runs in libgk_cuda.so; nothing here computes.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .config import Params

MODES = {"parity": _lib.GK_MODE_PARITY, "fast": _lib.GK_MODE_FAST}


def _descs(p: Params, mode: int, device: int):
    gd = _lib.GridDesc(p.nx, p.ny, p.nz, p.ng, p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax)
    pd = _lib.PhysDesc()
    pd.gamma, pd.cfl = p.gamma, p.cfl
    pd.integrator, pd.rc_order = int(p.integrator), int(p.rc_order)
    for i in range(6):
        pd.bc[i] = int(p.bc[i])
    for i in range(3):
        pd.grav[i] = float(p.grav[i])
    pd.dfloor, pd.pfloor = p.dfloor, p.pfloor
    pd.stepmax = int(p.stepmax)
    pd.mode = int(mode)
    pd.device = int(device)
    return gd, pd


class Sim:
    """One problem on one GPU.  ``mode`` is ``"parity"`` (bit-identical to the
    reference built with strict IEEE flags) or ``"fast"``."""

    def __init__(self, params: Params, cons: Optional[np.ndarray] = None, mode: str = "parity",
                 device: int = 0):
        """Sim::Sim (sim.cpp:45-67) through gk_create; ``cons``, if given, is
        uploaded as a setup hook leaves Sim::cons (main.cpp:25-30)."""
        self.params = params
        self.mode = mode
        self._L = _lib.load()
        gd, pd = _descs(params, MODES[mode], device)
        h = ctypes.c_void_p()
        _lib.check(self._L.gk_create(ctypes.byref(gd), ctypes.byref(pd), ctypes.byref(h)))
        self.h = h
        if cons is not None:
            self.upload(cons)

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.gk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state -----------------------------------------------------------
    def upload(self, cons: np.ndarray) -> None:
        """Loads Sim::cons (reference layout, ghosts included) after a setup hook
        or between outputs (main.cpp:25-30); clears the dt log."""
        c = np.ascontiguousarray(cons, dtype=np.float64)
        if c.shape != self.params.shape:
            raise ValueError(f"state shape {c.shape} != {self.params.shape}")
        _lib.check(self._L.gk_upload_cons(self.h, c.ctypes.data_as(ctypes.c_void_p)), self.h)

    def download(self, out: Optional[np.ndarray] = None, planes_only: bool = False) -> np.ndarray:
        """The state in the reference layout.  planes_only leaves the planes the
        device does not hold (1D/2D: k != nghost) as they are in ``out``, and on
        the fused 2D path a z-momentum plane that was zero at upload too."""
        if out is None:
            out = np.empty(self.params.shape, dtype=np.float64)
            planes_only = False
        assert out.shape == self.params.shape and out.dtype == np.float64 and out.flags.c_contiguous
        fn = self._L.gk_download_planes if planes_only else self._L.gk_download_cons
        _lib.check(fn(self.h, out.ctypes.data_as(ctypes.c_void_p)), self.h)
        return out

    def floor_hits(self) -> Tuple[int, int]:
        """Cells whose density / pressure the floors repaired since the last upload."""
        d, p = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        _lib.check(self._L.gk_floor_hits(self.h, ctypes.byref(d), ctypes.byref(p)), self.h)
        return d.value, p.value

    def io_bytes(self) -> Tuple[int, int]:
        """Bytes the last upload and the last download moved across the bus."""
        up, down = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(self._L.gk_io_bytes(self.h, ctypes.byref(up), ctypes.byref(down)), self.h)
        return up.value, down.value

    # -- time loop -------------------------------------------------------
    def advance(self, dtoutput: float) -> Tuple[float, int, bool]:
        """Sim::Advance(dtoutput) (sim.cpp:69-117); returns (t, step, isContinue)."""
        t, step, cont = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self._L.gk_advance(self.h, float(dtoutput), ctypes.byref(t), ctypes.byref(step),
                                      ctypes.byref(cont)), self.h)
        return t.value, step.value, bool(cont.value)

    def run(self, tmax: Optional[float] = None, dtoutput: Optional[float] = None) -> None:
        """main.cpp:44-52 without the frame writes."""
        tmax = self.params.tmax if tmax is None else tmax
        dtoutput = self.params.dtoutput if dtoutput is None else dtoutput
        if not dtoutput or dtoutput <= 0:
            dtoutput = tmax
        t = self.get_time()
        while abs(tmax - t) > 1e-12 and self.is_continue:
            dtoutput = min(dtoutput, tmax - t)
            t, _, _ = self.advance(dtoutput)

    def run_steps(self, n: int) -> int:
        """n steps of the Sim::Advance loop body (sim.cpp:72-103) with no output
        time; returns the steps taken (fewer if stepmax ends the run)."""
        done = ctypes.c_int()
        _lib.check(self._L.gk_run_steps(self.h, int(n), ctypes.byref(done)), self.h)
        return done.value

    def enqueue_steps(self, n: int) -> None:
        """As run_steps, but returns once the steps are enqueued on ``stream``."""
        _lib.check(self._L.gk_enqueue_steps(self.h, int(n)), self.h)

    def _time(self):
        t, dt, step, cont = ctypes.c_double(), ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self._L.gk_get_time(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(step),
                                       ctypes.byref(cont)), self.h)
        return t.value, dt.value, step.value, bool(cont.value)

    def get_time(self) -> float:
        """Sim::GetTime (sim.hpp:43)."""
        return self._time()[0]

    def get_dt(self) -> float:
        """Sim::Getdt (sim.hpp:44)."""
        return self._time()[1]

    def get_step(self) -> int:
        """Sim::GetStep (sim.hpp:45)."""
        return self._time()[2]

    @property
    def is_continue(self) -> bool:
        """Sim::isContinue (sim.hpp:26)."""
        return self._time()[3]

    def set_time(self, t: float, step: int) -> None:
        """Sets the clock for a restart from a frame (no reference counterpart:
        t and step are private, sim.hpp:48-49)."""
        _lib.check(self._L.gk_set_time(self.h, float(t), int(step)), self.h)

    def dt_log(self) -> List[float]:
        """dt of every step since the last upload, at full precision (the values
        Sim::Advance prints, sim.cpp:100-103)."""
        n = ctypes.c_int()
        _lib.check(self._L.gk_dt_log(self.h, None, 0, ctypes.byref(n)), self.h)
        buf = np.empty(max(n.value, 1), dtype=np.float64)
        _lib.check(self._L.gk_dt_log(self.h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     n.value, ctypes.byref(n)), self.h)
        return buf[:n.value].tolist()

    def cmax(self) -> float:
        """EquationOfState::CalCmax seeded with 1e-16 (sim.cpp:77-78) of the
        current state."""
        c = ctypes.c_double()
        _lib.check(self._L.gk_cmax(self.h, ctypes.byref(c)), self.h)
        return c.value

    @property
    def path(self) -> str:
        """The device implementation selected: "generic", "fused2d", "stage3d"
        or "run1d" (the results are the same bits in parity mode)."""
        p = ctypes.c_int()
        _lib.check(self._L.gk_path(self.h, ctypes.byref(p)), self.h)
        return {0: "generic", 1: "fused2d", 2: "stage3d", 3: "run1d"}[p.value]

    def set_fixed_boundary(self, snapshot: Optional[np.ndarray], fix_inner: bool = False) -> None:
        """Data of the fixed (type 4) sides: the reference-layout state at
        enrollment (Boundary::EnrollFixedBoundaryData); fix_inner also resets
        the inner disk (FixedBDInner).  None removes them."""
        if snapshot is None:
            _lib.check(self._L.gk_set_fixed_boundary(self.h, None, 0), self.h)
            return
        a = np.ascontiguousarray(snapshot, dtype=np.float64)
        if a.shape != self.params.shape:
            raise ValueError(f"snapshot shape {a.shape} != {self.params.shape}")
        _lib.check(self._L.gk_set_fixed_boundary(self.h, a.ctypes.data_as(ctypes.c_void_p),
                                                 int(bool(fix_inner))), self.h)

    def set_point_gravity(self, masses: Sequence[Sequence[float]]) -> None:
        """Point masses as SourceTerm::EnrollPointGravity takes them, each
        (gm, x, y, z, rs); none, one, or two (a binary: the second orbits the
        first with the separation, angular speed and phase the reference's
        EnrollPointGravity computes)."""
        import math
        if len(masses) > 2:
            raise ValueError("at most two point masses")
        p = np.zeros(11)
        if masses:
            p[0:5] = masses[0]
        if len(masses) == 2:
            gm0, x0, y0, z0, _ = masses[0]
            gm, x, y, z, rs = masses[1]
            ab = math.sqrt((x - x0) * (x - x0) + (y - y0) * (y - y0) + (z - z0) * (z - z0))
            p[5:8] = (gm, z, rs)
            p[8] = math.sqrt((gm0 + gm) / (ab * ab * ab))
            p[9] = ab
            p[10] = math.atan2(y - y0, x - x0)
        _lib.check(self._L.gk_set_point_gravity(self.h, len(masses),
                                                p.ctypes.data_as(ctypes.c_void_p)), self.h)

    def set_immersed(self, ids: Optional[np.ndarray], ntar: Optional[np.ndarray] = None,
                     direction: Optional[np.ndarray] = None,
                     weights: Optional[np.ndarray] = None) -> None:
        """An immersed solid body as the table Boundary::SetupImmersedShell
        builds: ids int (3, n, 9) of shell cells (t = 0) and targets
        (reference indices i, j, k), ntar int (n,), direction (4, n) =
        cos(phi), sin(phi), cos(theta), sin(theta), weights (n, 9) =
        disGamma.  None removes the body."""
        if ids is None:
            _lib.check(self._L.gk_set_immersed(self.h, 0, None, None, None, None), self.h)
            return
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        n = ids.shape[1]
        ntar = np.ascontiguousarray(ntar, dtype=np.int32)
        direction = np.ascontiguousarray(direction, dtype=np.float64)
        weights = np.ascontiguousarray(weights, dtype=np.float64)
        if (ids.shape != (3, n, 9) or ntar.shape != (n,) or direction.shape != (4, n)
                or weights.shape != (n, 9)):
            raise ValueError("immersed table shapes: ids (3, n, 9), ntar (n,), direction (4, n), "
                             "weights (n, 9)")
        vp = ctypes.c_void_p
        _lib.check(self._L.gk_set_immersed(self.h, n, ids.ctypes.data_as(vp), ntar.ctypes.data_as(vp),
                                           direction.ctypes.data_as(vp),
                                           weights.ctypes.data_as(vp)), self.h)

    def set_tiling(self, threads: int, rows: int) -> None:
        """Tile shape of the fused 2D stage kernel (threads per CTA 64/128/256,
        rows per segment); see gaukuk_b200.autotune."""
        _lib.check(self._L.gk_set_tiling(self.h, int(threads), int(rows)), self.h)

    def graph_info(self) -> Tuple[int, int]:
        """(whole steps per graph launch, kernel launches per step)."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._L.gk_graph_info(self.h, ctypes.byref(a), ctypes.byref(b)), self.h)
        return a.value, b.value

    @property
    def stream(self) -> int:
        """The handle's CUDA stream (a cudaStream_t as an integer)."""
        s = ctypes.c_void_p()
        _lib.check(self._L.gk_stream(self.h, ctypes.byref(s)), self.h)
        return s.value or 0

    def profile(self, nsteps: int) -> Dict[str, Tuple[float, int]]:
        """Device milliseconds and launch counts per kernel class over nsteps
        un-graphed steps (CUDA events on the handle's stream)."""
        cap = 16
        names = ctypes.create_string_buffer(512)
        ms = (ctypes.c_double * cap)()
        cnt = (ctypes.c_int * cap)()
        n = ctypes.c_int()
        _lib.check(self._L.gk_profile_steps(self.h, int(nsteps), names, 512, ms, cnt, cap,
                                            ctypes.byref(n)), self.h)
        keys = names.value.decode().split(";") if n.value else []
        return {k: (ms[i], cnt[i]) for i, k in enumerate(keys)}
