"""gk_rk2_step_noalloc: the RK2 step for callers that cannot allocate device
memory while they run (their memory comes from their own pool or arena, or
their budget is fixed at start-up).  The caller owns the state; the library's
stage state and clock live in a fixed array inside the library.

Checked against the handle path (gk_create + gk_run_steps, which allocates)
on the same initial state, over two calls in a row: bit-identical state and
dt in parity mode, within the fast-mode tolerance (1e-12) in fast mode.
The file is named so that pytest collects it after every other test.
"""
import ctypes
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import problems
from helpers import active, rel_linf

pytestmark = pytest.mark.gpu

SLOTS = (0, 1, 2, 4, 3)  # device planes DEN, MTX, MTY, ENG, MTZ <- reference vars


def to_device_layout(p, cons):
    pitch = (p.lenx + 15) // 16 * 16
    out = np.zeros((5, p.leny, pitch))
    for s, v in enumerate(SLOTS):
        out[s, :, :p.lenx] = cons[v, p.ng]
    return out


def active_from_device_layout(p, dev):
    a = np.zeros((5, 1, p.ny, p.nx))
    g = p.ng
    for s, v in enumerate(SLOTS):
        a[v, 0] = dev[s, g:g + p.ny, g:g + p.nx]
    return a


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_noalloc_step_matches_handle_over_two_calls(mode):
    import torch
    from gaukuk_b200 import _lib
    from gaukuk_b200.sim import MODES, Sim, _descs

    p, c = problems.kh(150, ny=130, seed=7)
    p = dataclasses.replace(p, stepmax=-1)
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
            assert abs(dt.value - ref_dt) <= 1e-12 * ref_dt, call
            errs = rel_linf(got, want)
            assert max(errs[v] for v in (0, 1, 2, 4)) <= 1e-12, (call, errs)
    ref.close()


def test_noalloc_rejects_oversized_grid():
    from gaukuk_b200 import _lib
    from gaukuk_b200.sim import MODES, _descs
    p, _ = problems.kh(8)
    p = dataclasses.replace(p, nx=2048, ny=2048)
    gd, pd = _descs(p, MODES["parity"], 0)
    L = _lib.load()
    rc = L.gk_rk2_step_noalloc(ctypes.byref(gd), ctypes.byref(pd), ctypes.c_void_p(1), 1.0,
                               None, None)
    assert rc == -1  # GK_ERR_INVALID, before any device work
