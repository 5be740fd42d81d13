"""Run parameters and the reference's ``.in`` file format.

The ``.in`` reader follows ``Config::loadFromFile`` (src/utils/read_config.cpp:18-46):
blank lines and lines starting with ``#`` are skipped, the first ``=`` becomes a
space, and the line is read as ``key value`` where the value is a number
(``Real``); trailing text after the number is ignored.  A missing key reads as
its default (``Config::get``, read_config.cpp:48-50), 0 unless stated.
"""
from __future__ import annotations

import dataclasses
import re
from typing import Dict, Optional

# Boundary type ids (boundary.cpp:13-125)
BC_COPY, BC_PERIODIC, BC_REFLECTIVE, BC_OUTFLOW, BC_FIXED = 0, 1, 2, 3, 4

_NUM = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")


def parse_in_text(text: str) -> Dict[str, float]:
    """Parse ``.in`` text into a key -> float dict, as Config::loadFromFile does."""
    data: Dict[str, float] = {}
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        line = line.replace("=", " ", 1)
        parts = line.split()
        if len(parts) < 2:
            continue
        m = _NUM.match(parts[1])
        if not m:
            continue
        data[parts[0]] = float(m.group(0))
    return data


def load_in(path: str) -> Dict[str, float]:
    with open(path, "r") as f:
        return parse_in_text(f.read())


@dataclasses.dataclass
class Params:
    """Everything the finite-volume update reads from the ``.in`` file.

    Field meanings follow the reference: Grid (grid.hpp:18-41), Domain
    (sim.cpp:16-42), Sim::Sim (sim.cpp:45-67), EquationOfState
    (adiabatic.cpp:12-16), Boundary (boundary.cpp:13-20), and the gravity
    vector a setup hook enrolls (source.cpp:23-31).
    """

    nx: int
    ny: int = 1
    nz: int = 1
    ng: int = 2
    xmin: float = 0.0
    xmax: float = 1.0
    ymin: float = 0.0
    ymax: float = 1.0
    zmin: float = 0.0
    zmax: float = 1.0
    gamma: float = 1.4
    cfl: float = 0.4
    integrator: int = 2
    rc_order: int = 2
    bc: tuple = (1, 1, 1, 1, 1, 1)
    grav: tuple = (0.0, 0.0, 0.0)
    dfloor: float = 1e-16
    pfloor: float = 1e-16
    stepmax: int = -1
    tmax: float = 0.0
    dtoutput: float = 0.0

    @property
    def lenx(self) -> int:
        return self.nx + 2 * self.ng

    @property
    def leny(self) -> int:
        return self.ny + 2 * self.ng

    @property
    def lenz(self) -> int:
        return self.nz + 2 * self.ng

    @property
    def shape(self):
        """Reference TArray shape of cons: (NVar, lenz, leny, lenx)."""
        return (5, self.lenz, self.leny, self.lenx)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def ndim(self) -> int:
        if self.nz > 1:
            return 3
        return 2 if self.ny > 1 else 1

    @classmethod
    def from_in(cls, data: Dict[str, float]) -> "Params":
        g = lambda k, d=0.0: data.get(k, d)  # noqa: E731
        return cls(
            nx=int(g("NX")), ny=int(g("NY")), nz=int(g("NZ")), ng=int(g("NGhost")),
            xmin=g("xmin"), xmax=g("xmax"), ymin=g("ymin"), ymax=g("ymax"),
            zmin=g("zmin"), zmax=g("zmax"), gamma=g("gamma"), cfl=g("CFL"),
            integrator=int(g("integrator", 2)), rc_order=int(g("RcOrder", 1)),
            bc=tuple(int(g(k)) for k in ("xleft", "xright", "yleft", "yright", "zleft", "zright")),
            grav=(g("gx"), g("gy"), g("gz")),
            stepmax=int(g("stepmax", -1)), tmax=g("tmax"), dtoutput=g("dtoutput"),
        )

    def to_in_text(self, extra: Optional[Dict[str, float]] = None) -> str:
        """Render as an ``.in`` file the reference (and this package) can read."""
        kv = {
            "gamma": self.gamma, "CFL": self.cfl, "integrator": self.integrator,
            "RcOrder": self.rc_order, "tmax": self.tmax, "dtoutput": self.dtoutput,
            "stepmax": self.stepmax, "dataType": 0,
            "xmin": self.xmin, "xmax": self.xmax, "ymin": self.ymin, "ymax": self.ymax,
            "zmin": self.zmin, "zmax": self.zmax,
            "NX": self.nx, "NY": self.ny, "NZ": self.nz, "NGhost": self.ng,
            "xleft": self.bc[0], "xright": self.bc[1], "yleft": self.bc[2],
            "yright": self.bc[3], "zleft": self.bc[4], "zright": self.bc[5],
            "gx": self.grav[0], "gy": self.grav[1], "gz": self.grav[2],
        }
        if extra:
            kv.update(extra)
        return "".join(f"{k} = {v!r}\n" for k, v in kv.items())
