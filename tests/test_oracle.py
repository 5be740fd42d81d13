"""The CPU oracle (oracle/gk_oracle.c) against the reference.

* golden vectors in tests/golden/ were produced by the reference built from
  its own sources (tests/golden/make_golden.py); the oracle must reproduce
  them bit for bit, dt sequence included;
* when the reference build is present (oracle/_ref), the oracle is also run
  side by side with it on fresh cases.
"""
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import problems
from gaukuk_b200.config import Params
from helpers import active, golden_cases, load_golden

gk_oracle = pytest.importorskip("gk_oracle")


@pytest.mark.parametrize("name", sorted(golden_cases()))
def test_oracle_matches_golden(name):
    p, cons, final, dts = load_golden(name)
    o = gk_oracle.OracleSim(p, cons)
    got_dts = o.run(p.tmax, p.dtoutput)
    assert got_dts == dts
    assert np.array_equal(active(p, o.get_cons()), final)


def _ref_cases():
    p, c = problems.kh(40, ny=36, seed=3)
    yield "kh_rk2", dataclasses.replace(p, stepmax=30), c
    p, c = problems.kh(33, ny=29, integrator=3, seed=1)
    yield "kh_rk3_odd", dataclasses.replace(p, stepmax=20, bc=(2, 3, 0, 1, 1, 1)), c
    p, c = problems.sod(200, bc=3)
    yield "sod_outflow", p, c
    p, c = problems.rt(24, 72)
    yield "rt", dataclasses.replace(p, stepmax=25), c
    p = Params(nx=12, ny=10, nz=9, bc=(3, 2, 1, 1, 2, 0), integrator=2, rc_order=1, tmax=1.0,
               dtoutput=1.0, stepmax=6)
    yield "box_rc1", p, problems.random_smooth(p, seed=2, with_vz=True)


@pytest.mark.skipif(not gk_oracle.reference_available("strict"), reason="reference build absent")
@pytest.mark.parametrize("case", list(_ref_cases()), ids=lambda c: c[0])
def test_oracle_matches_reference_build(case):
    _, p, c = case
    ref, ref_dts, _ = gk_oracle.run_reference(p, c, flavour="strict")
    o = gk_oracle.OracleSim(p, c)
    dts = o.run(p.tmax, p.dtoutput)
    assert dts == ref_dts
    assert np.array_equal(active(p, o.get_cons()), active(p, ref))


@pytest.mark.skipif(not gk_oracle.reference_available("fast"), reason="reference build absent")
def test_fast_reference_within_tolerance_of_strict():
    """The reference's own Makefile flags (-ffast-math) differ from strict
    IEEE by rounding only: far below the 1e-12 contract."""
    p, c = problems.kh(64)
    p = dataclasses.replace(p, stepmax=100)
    a, _, _ = gk_oracle.run_reference(p, c, flavour="strict")
    b, _, _ = gk_oracle.run_reference(p, c, flavour="fast")
    for v in (0, 1, 2, 4):
        x, y = active(p, a)[v], active(p, b)[v]
        assert np.max(np.abs(x - y)) / np.max(np.abs(x)) < 1e-12


def test_hllc_batch_symmetry():
    """HLLC of a state with itself is the exact Euler flux (hllc.cpp:22-101)."""
    rng = np.random.default_rng(0)
    n = 1000
    w = np.stack([rng.uniform(0.5, 2, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n),
                  rng.uniform(-1, 1, n), rng.uniform(0.5, 2, n)])
    f = gk_oracle.hllc_batch(w, w, 1, 1.4)
    rho, vx, vy, vz, p = w
    e = p / 0.4 + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    np.testing.assert_allclose(f[0], rho * vx, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(f[1], rho * vx * vx + p, rtol=1e-13)
    np.testing.assert_allclose(f[4], (e + p) * vx, rtol=1e-12, atol=1e-15)


def _random_faces(n, seed):
    rng = np.random.default_rng(seed)
    def one():
        return np.stack([rng.uniform(0.2, 3, n), rng.uniform(-2, 2, n), rng.uniform(-1, 1, n),
                         rng.uniform(-1, 1, n), rng.uniform(0.2, 3, n)])
    return one(), one()


def test_hllc_mirror_symmetry():
    """Reflecting a face (sides swapped, normal velocity negated) negates the
    mass, tangential-momentum and energy fluxes and keeps the normal-momentum
    flux (hllc.cpp:22-101 is symmetric up to rounding)."""
    wl, wr = _random_faces(2000, 1)
    f = gk_oracle.hllc_batch(wl, wr, 1, 1.4)
    ml, mr = wr.copy(), wl.copy()
    ml[1] *= -1
    mr[1] *= -1
    g = gk_oracle.hllc_batch(ml, mr, 1, 1.4)
    scale = np.abs(f).max(axis=1, keepdims=True)
    for v, sign in ((0, -1), (1, 1), (2, -1), (3, -1), (4, -1)):
        assert np.max(np.abs(g[v] - sign * f[v]) / scale[v]) < 1e-13, v


def test_hllc_resolves_an_isolated_contact():
    """Equal pressure and normal velocity, different density and tangential
    velocity: HLLC (unlike HLL) returns the upwind side's physical flux."""
    wl, wr = _random_faces(2000, 2)
    wr[1], wr[4] = wl[1], wl[4]
    f = gk_oracle.hllc_batch(wl, wr, 1, 1.4)
    up = np.where(wl[1] >= 0, wl, wr)
    rho, vx, vy, vz, p = up
    e = p / 0.4 + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    exact = np.stack([rho * vx, rho * vx * vx + p, rho * vx * vy, rho * vx * vz, (e + p) * vx])
    scale = np.abs(exact).max(axis=1, keepdims=True)
    assert np.max(np.abs(f - exact) / scale) < 1e-12


def test_vanleer_limiter():
    a = np.array([1.0, -1.0, 2.0, 0.0, -3.0])
    b = np.array([1.0, 2.0, 2.0, 5.0, -1.0])
    np.testing.assert_array_equal(gk_oracle.vanleer_batch(a, b), [1.0, 0.0, 2.0, 0.0, -1.5])


def test_conservation_periodic_kh():
    """Periodic KH conserves mass and energy to round-off (the reference's
    own check, plot_kh.py:41-83)."""
    p, c = problems.kh(48)
    o = gk_oracle.OracleSim(dataclasses.replace(p, stepmax=50), c)
    m0 = active(p, c).sum(axis=(1, 2, 3))
    o.run(p.tmax, p.dtoutput)
    m1 = active(p, o.get_cons()).sum(axis=(1, 2, 3))
    assert abs(m1[0] - m0[0]) / m0[0] < 1e-14
    assert abs(m1[4] - m0[4]) / m0[4] < 1e-14


# ------------------------------------------------------------------ exact Riemann solution (Sod)
def _riemann():
    return pytest.importorskip("riemann_exact")


SOD_L, SOD_R = (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)


def test_exact_riemann_star_state_matches_toro():
    """Toro (2009) Table 4.3, Test 1 (the Sod problem): p* 0.30313,
    u* 0.92745, rho*L 0.42632, rho*R 0.26557."""
    rx = _riemann()
    ps, us = rx.star_state(SOD_L, SOD_R)
    rl, rr = rx.star_densities(SOD_L, SOD_R)
    assert abs(ps - 0.30313) < 5e-6 and abs(us - 0.92745) < 5e-6
    assert abs(rl - 0.42632) < 5e-6 and abs(rr - 0.26557) < 5e-6


def test_exact_sod_solution_conserves():
    rx = _riemann()
    n = 400
    xl = np.arange(n) / n
    rho, m, e = rx.cell_average(xl, xl + 1.0 / n, 0.2, 0.5, SOD_L, SOD_R, sub=256)
    # the waves stay inside [0, 1] up to t = 0.2; flux in = flux out = p at the walls
    assert abs(rho.mean() - 0.5625) < 1e-4
    assert abs(e.mean() - 1.375) < 1e-4


def test_sod_converges_to_the_exact_solution():
    """The oracle's Sod run (PLM + HLLC + RK2, CFL 0.4, outflow) against the
    exact cell averages at t = 0.2: L1(rho) about 1.8e-3 at 256 cells,
    shrinking with resolution; mass exact."""
    rx = _riemann()
    from gaukuk_b200 import problems
    errs = []
    for n in (256, 512):
        p, c = problems.sod(n)
        o = gk_oracle.OracleSim(p, c)
        o.run(0.2, 0.2)
        a = o.get_cons()[:, p.ng, p.ng, p.ng:p.ng + n]
        xl = np.arange(n) / n
        rho, m, e = rx.cell_average(xl, xl + 1.0 / n, o.time, 0.5, SOD_L, SOD_R)
        errs.append(np.abs(a[0] - rho).mean())
        assert abs(a[0].mean() - 0.5625) < 1e-14
    assert errs[0] < 2.5e-3 and errs[1] < 0.75 * errs[0], errs
