"""The 1D run in one CTA (path 3, k_run1d): every step's ghost fill,
stages, CFL maximum and epilogue in one launch, many steps per launch.
Against the generic path (GK_RUN1D=0 at handle creation) on the same
state: state (ghosts included) and dt sequence bit for bit in parity mode,
within 1e-12 in fast mode; Sod against the oracle, and the largest row the
path takes (1020 cells).  Grids past that row length take the generic
path."""
import dataclasses
import os

import numpy as np
import pytest

from gaukuk_b200 import problems
from gaukuk_b200.config import BC_COPY, BC_OUTFLOW, BC_PERIODIC, BC_REFLECTIVE
from helpers import active

pytestmark = pytest.mark.gpu


def _case(name):
    if name == "sod_outflow_rk2":
        return problems.sod(256)
    if name == "sod_copy_rk3":
        return problems.sod(200, integrator=3, bc=BC_COPY)
    if name == "sod_reflective_euler":
        p, c = problems.sod(128, integrator=1, bc=BC_REFLECTIVE)
        return dataclasses.replace(p, cfl=0.2), c
    if name == "sod_first_order_periodic":
        p, c = problems.sod(96, bc=BC_PERIODIC)
        return dataclasses.replace(p, rc_order=1), c
    if name == "random_vz":  # transverse velocities (vz != 0: the z-momentum terms)
        p = problems.Params(nx=300, ny=1, nz=1, integrator=2, tmax=1.0, dtoutput=1.0,
                            bc=(BC_OUTFLOW, BC_REFLECTIVE) + (BC_PERIODIC,) * 4)
        return p, problems.random_smooth(p, seed=5, with_vz=True)
    if name == "longest_row":
        return problems.sod(1020)
    raise KeyError(name)


def _run(p, c, mode, generic, steps):
    from gaukuk_b200.sim import Sim
    old = os.environ.get("GK_RUN1D")
    os.environ["GK_RUN1D"] = "0" if generic else "1"
    try:
        s = Sim(dataclasses.replace(p, stepmax=steps), c, mode=mode)
    finally:
        if old is None:
            del os.environ["GK_RUN1D"]
        else:
            os.environ["GK_RUN1D"] = old
    with s:
        s.run(p.tmax, p.dtoutput)
        return s.download(), s.dt_log(), s.path


CASES = ["sod_outflow_rk2", "sod_copy_rk3", "sod_reflective_euler", "sod_first_order_periodic",
         "random_vz", "longest_row"]


@pytest.mark.parametrize("mode", ["parity", "fast"])
@pytest.mark.parametrize("case", CASES)
def test_one_cta_run_matches_the_generic_path(case, mode):
    p, c = _case(case)
    steps = 150
    a, da, pa = _run(p, c, mode, generic=False, steps=steps)
    b, db, pb = _run(p, c, mode, generic=True, steps=steps)
    assert pa == "run1d" and pb == "generic"
    assert 50 <= len(da) == len(db) <= steps  # the step cap, or the end time first
    if mode == "parity":
        assert da == db
        assert np.array_equal(a, b)
    else:
        for v in range(5):
            scale = max(float(np.max(np.abs(b[v]))), 1e-300)
            assert float(np.max(np.abs(a[v] - b[v]))) <= 1e-12 * scale, v
        assert max(abs(x - y) / y for x, y in zip(da, db)) <= 1e-12


def test_sod_on_the_one_cta_path_matches_the_oracle():
    """Sod 256 to t = 0.2 (280 steps), parity mode: the oracle's bits."""
    gk_oracle = pytest.importorskip("gk_oracle")
    from gaukuk_b200.sim import Sim
    p, c = problems.sod(256)
    o = gk_oracle.OracleSim(p, c)
    odts = o.run(p.tmax, p.dtoutput)
    with Sim(p, c, mode="parity") as s:
        assert s.path == "run1d"
        s.run(p.tmax, p.dtoutput)
        assert s.dt_log() == odts
        assert np.array_equal(active(p, s.download()), active(p, o.get_cons()))


def test_rows_past_1024_take_the_generic_path():
    from gaukuk_b200.sim import Sim
    p, c = problems.sod(1021)
    with Sim(p, c, mode="parity") as s:
        assert s.path == "generic"
