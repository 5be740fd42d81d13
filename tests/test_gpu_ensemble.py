"""Ensembles (persistent launch over a tile table, captured graph): every
instance must equal the same problem run alone, bit for bit in parity mode,
dt sequence included, whatever the tile shape.  In fast mode the compiler
may contract the ensemble kernel's arithmetic differently from the
single-problem kernel's, so there the contract is the fast-mode tolerance."""
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import problems
from helpers import active, rel_linf

pytestmark = pytest.mark.gpu


def _instances():
    out = []
    for i, (nx, ny) in enumerate([(64, 64), (48, 40), (130, 70), (96, 72), (20, 300), (257, 33)]):
        p, c = problems.kh(nx, ny=ny, seed=i, rho_in=1.5 + 0.4 * i, half_width=0.2 + 0.015 * i)
        out.append((dataclasses.replace(p, tmax=0.06, dtoutput=0.03), c))
    return out


def _solo(p, c, mode):
    from gaukuk_b200.sim import Sim
    s = Sim(p, c, mode=mode)
    s.run(p.tmax, p.dtoutput)
    return active(p, s.download()), s.dt_log()


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_ensemble_equals_solo_runs(mode):
    from gaukuk_b200.ensemble import Ensemble
    from gaukuk_b200.sim import Sim
    inst = _instances()
    sims = [Sim(p, c, mode=mode) for p, c in inst]
    ens = Ensemble(sims)
    ens.run(0.06, 0.03)
    for (p, c), s in zip(inst, sims):
        ref, ref_dts = _solo(p, c, mode)
        dts = s.dt_log()
        if mode == "parity":
            assert dts == ref_dts
            assert np.array_equal(active(p, s.download()), ref)
        else:
            assert len(dts) == len(ref_dts)
            np.testing.assert_allclose(dts, ref_dts, rtol=1e-12)
            errs = rel_linf(active(p, s.download()), ref)
            assert max(errs[v] for v in (0, 1, 2, 4)) <= 1e-12, errs


@pytest.mark.parametrize("threads,rows", [(64, [3, 5, 7, 4, 9, 2]), (256, [16] * 6), (128, [32] * 6)])
def test_ensemble_tiling_does_not_change_results(threads, rows):
    from gaukuk_b200.ensemble import Ensemble
    from gaukuk_b200.sim import Sim
    inst = _instances()
    sims = [Sim(p, c, mode="parity") for p, c in inst]
    ens = Ensemble(sims, threads=threads, rows=rows)
    ens.run_steps(5)
    for (p, c), s in zip(inst, sims):
        solo = Sim(p, c, mode="parity")
        solo.run_steps(5)
        assert s.dt_log() == solo.dt_log()
        assert np.array_equal(active(p, s.download()), active(p, solo.download()))


@pytest.mark.parametrize("threads,rows", [(64, 5), (256, 3), (128, 64)])
def test_single_problem_tiling_does_not_change_results(threads, rows):
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(150, ny=90, seed=2)
    a = Sim(p, c, mode="parity")
    b = Sim(p, c, mode="parity")
    b.set_tiling(threads, rows)
    a.run_steps(6)
    b.run_steps(6)
    assert a.dt_log() == b.dt_log()
    assert np.array_equal(active(p, a.download()), active(p, b.download()))


def test_autotuner_applies_a_candidate():
    from gaukuk_b200 import autotune
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(256, seed=1)
    s = Sim(p, c, mode="fast")
    th, rows, ms = autotune.tune_single(s, steps=2, use_cache=False)
    assert th in autotune.THREADS and rows in autotune.ROWS and ms > 0


def test_ensemble_refuses_fixed_sides_without_data():
    """An instance's physics is copied when the ensemble is made, so a
    handle with a fixed (type 4) side must have its data set first: without
    them creation fails with a state error; with them the ensemble runs and
    equals the same problem run alone."""
    from gaukuk_b200._lib import GkError
    from gaukuk_b200.ensemble import Ensemble
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(64, seed=2)
    p = dataclasses.replace(p, bc=(4, 4) + tuple(p.bc[2:]), tmax=0.03, dtoutput=0.03)
    s = Sim(p, c, mode="parity")
    with pytest.raises(GkError) as e:
        Ensemble([s])
    assert e.value.code == -5
    s.set_fixed_boundary(c)
    Ensemble([s]).run(p.tmax)
    got = active(p, s.download())
    ref = Sim(p, c, mode="parity")
    ref.set_fixed_boundary(c)
    ref.run(p.tmax, p.dtoutput)
    assert np.array_equal(got, active(p, ref.download()))
