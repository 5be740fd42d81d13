"""One 2D grid split into y-slabs (include/gaukuk_cuda.h, gk_slabs_*).

``Slabs(params, cons, nslab)`` runs the slabs in this process (on one GPU,
exchanging their ghost rows through device copies); ``DistSlabs`` runs one
slab per process of a ``torch.distributed`` job, exchanging through NCCL.
Both keep ``Sim``'s interface -- ``advance(dtoutput)`` is Sim::Advance of the
whole grid (sim.cpp:69-117), states cross in the reference layout of the
whole grid -- and both give the undivided grid's results bit for bit: every
ghost row a slab reads is the row the whole grid would hold there, and every
slab takes the whole grid's dt (the CFL maximum is taken over all slabs).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Tuple

import numpy as np

from . import _lib
from .config import Params
from .sim import MODES, _descs


def layout(ny: int, nslab: int, k: int, periodic: bool) -> Tuple[int, int, int, int]:
    """(first active row, rows, lower neighbour, upper neighbour) of slab k;
    a neighbour of -1 is a side of the grid.  Host only (no device needed)."""
    L = _lib.load()
    out = [ctypes.c_int() for _ in range(4)]
    _lib.check(L.gk_slab_layout(int(ny), int(nslab), int(k), int(bool(periodic)),
                                *[ctypes.byref(o) for o in out]))
    return tuple(o.value for o in out)


def exchange_plan(nslab: int, k: int, periodic: bool) -> List[Tuple[int, int]]:
    """The library's NCCL calls for one halo exchange of slab k, in order:
    (kind, peer) with kind 0 send top rows, 1 receive lower ghosts, 2 send
    bottom rows, 3 receive upper ghosts.  Host only."""
    L = _lib.load()
    ops = (ctypes.c_int * 8)()
    n = ctypes.c_int()
    _lib.check(L.gk_slab_exchange_plan(int(nslab), int(k), int(bool(periodic)), ops,
                                       ctypes.byref(n)))
    return [(ops[2 * o], ops[2 * o + 1]) for o in range(n.value)]


class _SlabsBase:
    def __init__(self, params: Params):
        self.params = params
        self._L = _lib.load()
        self.g = None

    def _check(self, rc: int) -> None:
        if rc != _lib.GK_OK:
            msg = self._L.gk_slabs_last_error(self.g).decode() if self.g else ""
            raise _lib.GkError(rc, f"{self._L.gk_strerror(rc).decode()}: {msg}")

    def close(self) -> None:
        if getattr(self, "g", None):
            self._L.gk_slabs_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, cons: np.ndarray) -> None:
        c = np.ascontiguousarray(cons, dtype=np.float64)
        if c.shape != self.params.shape:
            raise ValueError(f"state shape {c.shape} != {self.params.shape}")
        self._check(self._L.gk_slabs_upload_cons(self.g, c.ctypes.data_as(ctypes.c_void_p)))

    def download(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """This process's rows of the whole grid (all rows for ``Slabs``);
        other rows of ``out`` are left as they are (zero in a new array)."""
        if out is None:
            out = np.zeros(self.params.shape, dtype=np.float64)
        self._check(self._L.gk_slabs_download_cons(self.g, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def advance(self, dtoutput: float) -> Tuple[float, int, bool]:
        t, step, cont = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        self._check(self._L.gk_slabs_advance(self.g, float(dtoutput), ctypes.byref(t),
                                             ctypes.byref(step), ctypes.byref(cont)))
        self._t, self._cont = t.value, bool(cont.value)
        return t.value, step.value, bool(cont.value)

    def run(self, tmax: float, dtoutput: Optional[float] = None) -> None:
        """main.cpp's output loop (main.cpp:44-52) without the writes, from
        the time of the last advance (0 for a new grid)."""
        dtoutput = tmax if not dtoutput else dtoutput
        t, cont = getattr(self, "_t", 0.0), getattr(self, "_cont", True)
        while abs(tmax - t) > 1e-12 and cont:
            t, _, cont = self.advance(min(dtoutput, tmax - t))

    def run_steps(self, n: int) -> int:
        done = ctypes.c_int()
        self._check(self._L.gk_slabs_run_steps(self.g, int(n), ctypes.byref(done)))
        return done.value

    def dt_log(self) -> List[float]:
        cap = 1 << 20
        buf = np.empty(cap, dtype=np.float64)
        n = ctypes.c_int()
        self._check(self._L.gk_slabs_dt_log(self.g, buf.ctypes.data_as(_lib._dp), cap,
                                            ctypes.byref(n)))
        return buf[:min(n.value, cap)].tolist()

    def info(self):
        a, b, c, d = (ctypes.c_int() for _ in range(4))
        self._check(self._L.gk_slabs_info(self.g, ctypes.byref(a), ctypes.byref(b),
                                          ctypes.byref(c), ctypes.byref(d)))
        return {"local_slabs": a.value, "first": b.value, "first_row": c.value,
                "rows": d.value}


class Slabs(_SlabsBase):
    """``nslab`` y-slabs of one grid in this process (one device)."""

    def __init__(self, params: Params, cons: Optional[np.ndarray], nslab: int,
                 mode: str = "parity", device: int = 0):
        super().__init__(params)
        gd, pd = _descs(params, MODES[mode], device)
        g = ctypes.c_void_p()
        _lib.check(self._L.gk_slabs_create(ctypes.byref(gd), ctypes.byref(pd), int(nslab),
                                           ctypes.byref(g)))
        self.g = g
        if cons is not None:
            self.upload(cons)


def nccl_id_broadcast(dist, make_id=None) -> bytes:
    """A 128-byte NCCL unique id made on rank 0 and broadcast to every rank
    of the torch.distributed group ``dist`` (any backend)."""
    if dist.get_rank() == 0:
        if make_id is None:
            buf = ctypes.create_string_buffer(128)
            _lib.check(_lib.load().gk_slabs_nccl_id(buf))
            raw = buf.raw
        else:
            raw = make_id()
    else:
        raw = None
    box = [raw]
    dist.broadcast_object_list(box, src=0)
    if not isinstance(box[0], (bytes, bytearray)) or len(box[0]) != 128:
        raise RuntimeError("NCCL id broadcast failed")
    return bytes(box[0])


class DistSlabs(_SlabsBase):
    """One y-slab per process of the initialised torch.distributed group
    (slab index = rank), exchanging through NCCL on device ``device``."""

    def __init__(self, params: Params, cons: Optional[np.ndarray], dist, mode: str = "parity",
                 device: int = 0):
        super().__init__(params)
        rank, world = dist.get_rank(), dist.get_world_size()
        nid = nccl_id_broadcast(dist)
        gd, pd = _descs(params, MODES[mode], device)
        g = ctypes.c_void_p()
        idbuf = ctypes.create_string_buffer(nid, 128)
        _lib.check(self._L.gk_slabs_create_nccl(ctypes.byref(gd), ctypes.byref(pd), int(world),
                                                int(rank), idbuf, ctypes.byref(g)))
        self.g = g
        if cons is not None:
            self.upload(cons)
