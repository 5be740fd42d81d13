"""The benchmark configurations at their stated sizes, 100 steps, against the
reference itself (oracle/_ref/ref_strict: the reference's sources compiled
with strict IEEE flags, OpenMP on every host core).

* Kelvin-Helmholtz 4096^2, PLM + HLLC + RK2 (the throughput workload);
* Rayleigh-Taylor 1024x3072, RK3 + constant gravity, reflecting walls;
* Kelvin-Helmholtz 256^2 in parity mode;
* one instance of each grid size of the ensemble configuration (128^2,
  256^2, 512^2, parameters drawn by its generator), advanced together as an
  ensemble.

Parity mode: every active conserved value and every dt equal the
reference's bits.  Fast mode: at most 1e-12 relative L-infinity per
conserved variable, the momentum components measured against the momentum's
magnitude (max over cells of max(|mx|, |my|)): a component that starts at
exactly zero, as RT's x-momentum does, has a maximum far below the momentum
scale, and against its own maximum it shows the rounding of the pressure in
the normal-momentum flux (the test prints both).  The largest relative
deviation of the dt sequence from the reference's, also printed, is at most
DT_TOL: fast mode's dt values are close to the reference's, not equal to
them (FMA contraction and refined approximate roots change the last bits of
cmax).
"""
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import problems
from helpers import active, rel_linf

pytestmark = pytest.mark.gpu
gk_oracle = pytest.importorskip("gk_oracle")

FAST_TOL = 1e-12
DT_TOL = 1e-13
STEPS = 100


def _need_reference():
    if not gk_oracle.reference_available("strict"):
        pytest.skip("the reference build (oracle/_ref/ref_strict) is not here")


def _reference(p, c):
    """Final active state and dt log of the reference on (p, c), 100 steps."""
    _need_reference()
    p = dataclasses.replace(p, stepmax=STEPS)
    out, dts, stats = gk_oracle.run_reference(p, c, flavour="strict", timeout=3600.0)
    assert len(dts) == STEPS and stats["steps"] == STEPS
    return active(p, out), dts


def _device(p, c, mode):
    from gaukuk_b200.sim import Sim
    p = dataclasses.replace(p, stepmax=STEPS)
    with Sim(p, c, mode=mode) as s:
        s.run(p.tmax, p.dtoutput)
        return active(p, s.download()), s.dt_log(), s.path


def _check(name, mode, got, dts, ref, ref_dts, evolved):
    assert len(dts) == len(ref_dts) == STEPS
    if mode == "parity":
        assert dts == ref_dts, name
        assert np.array_equal(got, ref), name
        return
    errs = rel_linf(got, ref)
    mscale = max(float(np.max(np.abs(ref[1]))), float(np.max(np.abs(ref[2]))))
    scaled = list(errs)
    for v in (1, 2):
        scaled[v] = float(np.max(np.abs(got[v] - ref[v]))) / mscale
    dev = float(np.max(np.abs(np.array(dts) - np.array(ref_dts)) / np.array(ref_dts)))
    print(f"\n{name} fast: rel Linf per variable {['%.2e' % errs[v] for v in evolved]}, "
          f"momentum against its magnitude {scaled[1]:.2e} {scaled[2]:.2e}, "
          f"max rel dt deviation {dev:.2e}")
    assert max(scaled[v] for v in evolved) <= FAST_TOL, (name, scaled)
    assert dev <= DT_TOL, (name, dev)


KH2D = (0, 1, 2, 4)  # DEN, MTX, MTY, ENG (MTZ stays 0)


@pytest.fixture(scope="module")
def kh4096():
    p, c = problems.kh(4096)
    ref, ref_dts = _reference(p, c)
    return p, c, ref, ref_dts


@pytest.fixture(scope="module")
def rt1024x3072():
    p, c = problems.rt(1024, 3072)
    ref, ref_dts = _reference(p, c)
    return p, c, ref, ref_dts


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_kh4096_100_steps_against_reference(kh4096, mode):
    p, c, ref, ref_dts = kh4096
    got, dts, path = _device(p, c, mode)
    assert path == "fused2d"
    _check("KH 4096^2 RK2", mode, got, dts, ref, ref_dts, KH2D)


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_rt1024x3072_rk3_gravity_100_steps_against_reference(rt1024x3072, mode):
    p, c, ref, ref_dts = rt1024x3072
    assert p.integrator == 3 and p.grav[1] != 0
    got, dts, path = _device(p, c, mode)
    assert path == "fused2d"
    _check("RT 1024x3072 RK3 + gravity", mode, got, dts, ref, ref_dts, KH2D)


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_kh256_100_steps_against_reference(mode):
    p, c = problems.kh(256)
    ref, ref_dts = _reference(p, c)
    got, dts, _ = _device(p, c, mode)
    _check("KH 256^2 RK2", mode, got, dts, ref, ref_dts, KH2D)


def _ensemble_instances():
    """The first instance of each grid size that the ensemble
    configuration's generator draws (64 instances, seed 0)."""
    picked = {}
    for p, c, draw in problems.kh_ensemble(64, seed=0):
        picked.setdefault(draw["size"], (p, c, draw))
    assert sorted(picked) == [128, 256, 512]
    return [picked[n] for n in (128, 256, 512)]


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_ensemble_instances_of_each_size_against_reference(mode):
    from gaukuk_b200.ensemble import Ensemble
    from gaukuk_b200.sim import Sim
    inst = _ensemble_instances()
    sims = [Sim(dataclasses.replace(p, stepmax=STEPS), c, mode=mode) for p, c, _ in inst]
    ens = Ensemble(sims)
    ens.run_steps(STEPS)
    for (p, c, draw), s in zip(inst, sims):
        ref, ref_dts = _reference(p, c)
        _check(f"ensemble instance {draw['size']}^2 (ratio {draw['ratio']:.3f})", mode,
               active(p, s.download()), s.dt_log(), ref, ref_dts, KH2D)
    ens.close()
    for s in sims:
        s.close()
