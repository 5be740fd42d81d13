"""gk_rk2_step_noalloc: the RK2 step for callers that cannot allocate device
memory while they run (their memory comes from their own pool or arena, or
their budget is fixed at start-up).  The caller owns the state; the library's
stage state and clock live in a fixed array inside the library.

Checked against the handle path (gk_create + gk_run_steps, which allocates)
on the same initial state, over two calls in a row: bit-identical state and
dt in parity mode, within the fast-mode tolerance (1e-12) in fast mode.  The
cases cover periodic, reflective, outflow and copy sides, constant gravity
(whose first half kick the entry point applies before the stages) and the
largest grid the fixed array accepts; a grid one row larger, and fixed
(type 4) sides, are refused before any device work.
The file is named so that pytest collects it after every other test.
"""
import ctypes
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import problems
from gaukuk_b200.config import BC_COPY, BC_FIXED, BC_OUTFLOW, BC_PERIODIC, BC_REFLECTIVE
from helpers import active, rel_linf

pytestmark = pytest.mark.gpu

SLOTS = (0, 1, 2, 4, 3)  # device planes DEN, MTX, MTY, ENG, MTZ <- reference vars
SCRATCH_DOUBLES = 1 << 23  # the library's fixed stage array
GK_ERR_INVALID, GK_ERR_UNSUPPORTED = -1, -4

# The largest accepted grid: 5 planes x leny x pitch <= 2^23 doubles with
# nx = 1276 (lenx 1280 = pitch) and ny = 1306 (leny 1310).
LIMIT_NX, LIMIT_NY = 1276, 1306


def _pitch(p):
    return (p.lenx + 15) // 16 * 16


def to_device_layout(p, cons):
    out = np.zeros((5, p.leny, _pitch(p)))
    for s, v in enumerate(SLOTS):
        out[s, :, :p.lenx] = cons[v, p.ng]
    return out


def active_from_device_layout(p, dev):
    a = np.zeros((5, 1, p.ny, p.nx))
    g = p.ng
    for s, v in enumerate(SLOTS):
        a[v, 0] = dev[s, g:g + p.ny, g:g + p.nx]
    return a


def _case(name):
    if name == "kh_periodic":
        return problems.kh(150, ny=130, seed=7)
    if name == "rt_gravity":
        return problems.rt(64, 192, integrator=2)
    if name == "kh_outflow_copy":
        p, c = problems.kh(96, ny=80, seed=3)
        return dataclasses.replace(p, bc=(BC_OUTFLOW, BC_OUTFLOW, BC_COPY, BC_REFLECTIVE,
                                          BC_PERIODIC, BC_PERIODIC)), c
    if name == "kh_limit":
        return problems.kh(LIMIT_NX, ny=LIMIT_NY, seed=11)
    raise KeyError(name)


@pytest.mark.parametrize("mode", ["parity", "fast"])
@pytest.mark.parametrize("case", ["kh_periodic", "rt_gravity", "kh_outflow_copy", "kh_limit"])
def test_noalloc_step_matches_handle_over_two_calls(case, mode):
    import torch
    from gaukuk_b200 import _lib
    from gaukuk_b200.sim import MODES, Sim, _descs

    p, c = _case(case)
    p = dataclasses.replace(p, stepmax=-1)
    if case == "kh_limit":
        assert 5 * p.leny * _pitch(p) <= SCRATCH_DOUBLES < 5 * (p.leny + 1) * _pitch(p)
    ref = Sim(p, c, mode=mode)

    L = _lib.load()
    gd, pd = _descs(p, MODES[mode], 0)
    torch.cuda.set_device(0)
    state = torch.from_numpy(to_device_layout(p, c)).cuda().contiguous()
    for call in range(2):
        dt = ctypes.c_double()
        rc = L.gk_rk2_step_noalloc(ctypes.byref(gd), ctypes.byref(pd),
                                   ctypes.c_void_p(state.data_ptr()), float("inf"),
                                   ctypes.byref(dt), None)
        _lib.check(rc)
        assert ref.run_steps(1) == 1
        got = active_from_device_layout(p, state.cpu().numpy())
        want = active(p, ref.download())
        ref_dt = ref.dt_log()[-1]
        if mode == "parity":
            assert dt.value == ref_dt, call
            assert np.array_equal(got, want), call
        else:
            # fast mode is held to its own tolerance
            assert abs(dt.value - ref_dt) <= 1e-12 * ref_dt, call
            errs = rel_linf(got, want)
            assert max(errs[v] for v in (0, 1, 2, 4)) <= 1e-12, (call, errs)
    ref.close()


def test_noalloc_rejects_grid_one_row_over_the_limit():
    """One row more than the limit grid: four planes would still fit, five
    (the ghost fill writes MTZ's ghosts too) do not."""
    from gaukuk_b200 import _lib
    from gaukuk_b200.sim import MODES, _descs
    p, _ = problems.kh(8)
    p = dataclasses.replace(p, nx=LIMIT_NX, ny=LIMIT_NY + 1)
    assert 4 * p.leny * _pitch(p) <= SCRATCH_DOUBLES < 5 * p.leny * _pitch(p)
    gd, pd = _descs(p, MODES["parity"], 0)
    L = _lib.load()
    rc = L.gk_rk2_step_noalloc(ctypes.byref(gd), ctypes.byref(pd), ctypes.c_void_p(1), 1.0,
                               None, None)
    assert rc == GK_ERR_INVALID  # before any device work


def test_noalloc_refuses_fixed_sides():
    from gaukuk_b200 import _lib
    from gaukuk_b200.sim import MODES, _descs
    p, _ = problems.kh(32)
    p = dataclasses.replace(p, bc=(BC_FIXED,) + (BC_PERIODIC,) * 5)
    gd, pd = _descs(p, MODES["parity"], 0)
    L = _lib.load()
    rc = L.gk_rk2_step_noalloc(ctypes.byref(gd), ctypes.byref(pd), ctypes.c_void_p(1), 1.0,
                               None, None)
    assert rc == GK_ERR_UNSUPPORTED  # before any device work
