"""Ensembles of independent 2D problems advanced together on one GPU.

Each instance is a ``Sim`` (its own state, clock and dt); the ensemble runs
every RK stage of every instance as one persistent launch over a tile table,
with whole steps held in a CUDA graph (include/gaukuk_cuda.h, gk_ens_*).
Results equal those of running each instance alone.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

from . import _lib
from .sim import Sim


class Ensemble:
    def __init__(self, sims: Sequence[Sim], threads: Optional[int] = None,
                 rows: Optional[Sequence[int]] = None):
        self.sims = list(sims)
        self._L = _lib.load()
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h.value for s in self.sims])
        e = ctypes.c_void_p()
        _lib.check(self._L.gk_ens_create(arr, len(self.sims), ctypes.byref(e)))
        self.e = e
        if threads is not None or rows is not None:
            self.set_tiling(threads or 128, rows)

    def close(self):
        if getattr(self, "e", None):
            self._L.gk_ens_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != _lib.GK_OK:
            msg = self._L.gk_ens_last_error(self.e).decode() if self.e else ""
            raise _lib.GkError(rc, f"{self._L.gk_strerror(rc).decode()}: {msg}")

    def set_tiling(self, threads: int, rows: Optional[Sequence[int]] = None) -> None:
        r = None
        if rows is not None:
            r = (ctypes.c_int * len(self.sims))(*[int(x) for x in rows])
        self._check(self._L.gk_ens_set_tiling(self.e, int(threads), r))

    def advance(self, dtoutput: float) -> None:
        """Sim::Advance(dtoutput) on every instance, each from its own time."""
        self._check(self._L.gk_ens_advance(self.e, float(dtoutput)))

    def run(self, tmax: float, dtoutput: Optional[float] = None) -> None:
        """main.cpp's output loop for every instance (all share tmax)."""
        dtoutput = tmax if not dtoutput else dtoutput
        while True:
            ts = [s.get_time() for s in self.sims]
            live = [abs(tmax - t) > 1e-12 and s.is_continue for s, t in zip(self.sims, ts)]
            if not any(live):
                return
            # every live instance is at the same output time here
            step = min(dtoutput, min(tmax - t for t, l in zip(ts, live) if l))
            self.advance(step)

    def run_steps(self, n: int) -> None:
        self._check(self._L.gk_ens_run_steps(self.e, int(n)))

    def enqueue_steps(self, n: int) -> None:
        self._check(self._L.gk_ens_enqueue_steps(self.e, int(n)))

    def info(self):
        nt, th = ctypes.c_int(), ctypes.c_int()
        st = ctypes.c_void_p()
        self._check(self._L.gk_ens_info(self.e, ctypes.byref(nt), ctypes.byref(th),
                                        ctypes.byref(st)))
        return {"tiles": nt.value, "threads": th.value, "stream": st.value or 0}
