"""The reference's output frames, cons_XXXXX / prim_XXXXX, and restarts.

Format (reference src/utils/write_sim.cpp:14-58, read back by
pypkg/read_gaukuk.py:3-44): int32 sizeof(Real), Real t, int32 NVar, nx, ny,
nz, nGhost, the cell centres with ghosts (lenx, leny, lenz Reals), int32
size, then the whole array NVar x lenz x leny x lenx (ghosts and every z
plane included), native byte order.

A restart reads a cons_ frame back: ``restart_sim`` builds a Sim on the
frame's state and time (the C++ driver does the same with the input key
``restart = N``, Sim::ReadData).  Frames do not carry the step counter, so it
restarts at 0.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

from .config import Params


@dataclasses.dataclass
class Frame:
    t: float
    nvar: int
    nx: int
    ny: int
    nz: int
    ng: int
    xc: np.ndarray  # cell centres with ghosts
    yc: np.ndarray
    zc: np.ndarray
    data: np.ndarray  # (nvar, lenz, leny, lenx)


def read_frame(path: str) -> Frame:
    with open(path, "rb") as f:
        real = int(np.fromfile(f, np.int32, 1)[0])
        if real not in (4, 8):
            raise ValueError(f"{path}: unknown Real size {real}")
        dt = np.float64 if real == 8 else np.float32
        t = float(np.fromfile(f, dt, 1)[0])
        nvar, nx, ny, nz, ng = (int(v) for v in np.fromfile(f, np.int32, 5))
        lx, ly, lz = nx + 2 * ng, ny + 2 * ng, nz + 2 * ng
        xc, yc, zc = (np.fromfile(f, dt, n) for n in (lx, ly, lz))
        size = int(np.fromfile(f, np.int32, 1)[0])
        if size != nvar * lx * ly * lz:
            raise ValueError(f"{path}: array size {size} does not match the header")
        data = np.fromfile(f, dt, size)
        if data.size != size:
            raise ValueError(f"{path}: truncated")
    return Frame(t, nvar, nx, ny, nz, ng, xc, yc, zc, data.reshape(nvar, lz, ly, lx))


def cell_centres(p: Params):
    """Centres with ghosts as Domain builds them, in its order of operations
    (reference src/sim.cpp:36-41): lo - ng*d + 0.5*d + i*d."""
    out = []
    for n, lo, hi in ((p.nx, p.xmin, p.xmax), (p.ny, p.ymin, p.ymax), (p.nz, p.zmin, p.zmax)):
        d = (hi - lo) / n
        i = np.arange(n + 2 * p.ng, dtype=np.float64)
        out.append(((lo - p.ng * d) + 0.5 * d) + i * d)
    return out


def write_frame(path: str, p: Params, t: float, data: np.ndarray) -> None:
    """Writes a frame in the reference's format; `data` is a reference-layout
    array (5 x lenz x leny x lenx doubles)."""
    data = np.ascontiguousarray(data, dtype=np.float64)
    if data.shape != p.shape:
        raise ValueError(f"state shape {data.shape} != {p.shape}")
    xc, yc, zc = cell_centres(p)
    with open(path, "wb") as f:
        np.array([8], np.int32).tofile(f)
        np.array([t], np.float64).tofile(f)
        np.array([data.shape[0], p.nx, p.ny, p.nz, p.ng], np.int32).tofile(f)
        for c in (xc, yc, zc):
            np.asarray(c, np.float64).tofile(f)
        np.array([data.size], np.int32).tofile(f)
        data.tofile(f)


def restart_sim(p: Params, path: str, mode: str = "parity", device: Optional[int] = None):
    """A Sim on the state and time of the cons_ frame at `path`; the frame's
    grid must match `p`."""
    from .sim import Sim
    fr = read_frame(path)
    if (fr.nvar, fr.nx, fr.ny, fr.nz, fr.ng) != (p.shape[0], p.nx, p.ny, p.nz, p.ng):
        raise ValueError(f"{path}: its grid differs from the parameters'")
    kw = {} if device is None else {"device": device}
    s = Sim(p, fr.data, mode=mode, **kw)
    s.set_time(fr.t, 0)
    return s
