"""Parity of the CUDA path (libgk_cuda.so, through the C ABI) with the oracle.

Parity mode must equal the oracle exactly -- every active conserved value
(np.array_equal, so -0.0 == 0.0) and every dt.  Fast mode must stay within
1e-12 relative L-infinity per conserved variable after 100 steps, the
contract for the floating-point path.
"""
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import problems
from gaukuk_b200.config import Params
from helpers import active, golden_cases, load_golden, rel_linf

pytestmark = pytest.mark.gpu
gk_oracle = pytest.importorskip("gk_oracle")

FAST_TOL = 1e-12


def _sim(p, c, mode="parity"):
    from gaukuk_b200.sim import Sim
    return Sim(p, c, mode=mode)


def _oracle_run(p, c):
    o = gk_oracle.OracleSim(p, c)
    dts = o.run(p.tmax, p.dtoutput)
    return active(p, o.get_cons()), dts, o


@pytest.mark.parametrize("name", sorted(golden_cases()))
def test_golden_vectors_on_gpu(name):
    p, cons, final, dts = load_golden(name)
    s = _sim(p, cons)
    s.run(p.tmax, p.dtoutput)
    assert s.dt_log() == dts
    assert np.array_equal(active(p, s.download()), final)


def _cases():
    p, c = problems.kh(64, seed=1)
    yield "kh64_rk2", dataclasses.replace(p, stepmax=60), c
    p, c = problems.kh(130, ny=70, seed=2, integrator=3)
    yield "kh130x70_rk3", dataclasses.replace(p, stepmax=30), c
    p, c = problems.kh(50, ny=300, seed=4, rc_order=1)
    yield "kh50x300_rc1_tall", dataclasses.replace(p, stepmax=20), c
    p, c = problems.kh(40, ny=40, integrator=1, cfl=0.2)
    yield "kh40_euler", dataclasses.replace(p, stepmax=20), c
    for bcs in [(2, 2, 3, 3, 1, 1), (3, 0, 2, 1, 1, 1), (0, 0, 0, 0, 1, 1)]:
        p, c = problems.kh(37, ny=45, seed=5)
        yield f"kh_bc{''.join(map(str, bcs[:4]))}", dataclasses.replace(p, bc=bcs, stepmax=25), c
    p, c = problems.sod(256)
    yield "sod256", p, c
    p, c = problems.sod(256, integrator=3, bc=2)
    yield "sod256_rk3_reflect", p, c
    p, c = problems.rt(32, 96)
    yield "rt32x96_gravity", dataclasses.replace(p, stepmax=40), c
    p = Params(nx=16, ny=12, nz=10, bc=(1, 1, 2, 3, 0, 1), integrator=3, tmax=1.0, dtoutput=1.0,
               stepmax=10)
    yield "box16x12x10", p, problems.random_smooth(p, seed=3, with_vz=True)
    p = Params(nx=24, ny=20, nz=1, integrator=2, tmax=1.0, dtoutput=1.0, stepmax=15)
    yield "kh_with_vz", p, problems.random_smooth(p, seed=4, with_vz=True)
    p = Params(nx=30, ny=18, nz=14, bc=(1,) * 6, integrator=2, tmax=1.0, dtoutput=1.0, stepmax=12)
    yield "box30x18x14_rk2", p, problems.random_smooth(p, seed=6, with_vz=True)
    p = Params(nx=20, ny=16, nz=12, bc=(3, 2, 0, 1, 2, 3), integrator=2, rc_order=1, tmax=1.0,
               dtoutput=1.0, stepmax=10)
    yield "box20x16x12_rc1_bcs", p, problems.random_smooth(p, seed=7, with_vz=True)


@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: c[0])
def test_parity_mode_bitwise(case):
    _, p, c = case
    ref, ref_dts, _ = _oracle_run(p, c)
    s = _sim(p, c)
    s.run(p.tmax, p.dtoutput)
    assert s.dt_log() == ref_dts
    assert np.array_equal(active(p, s.download()), ref)


def test_paths_selected():
    p, c = problems.kh(32)
    assert _sim(p, c).path == "fused2d"
    s = _sim(p, c)
    s.set_point_gravity([(1.0, 0.0, 0.0, 0.0, 0.1)])  # point masses run on the generic path
    assert s.path == "generic"
    p, c = problems.sod(64)
    assert _sim(p, c).path == "run1d"  # a 1D row of up to 1024 cells: one CTA
    p, c = problems.sod(2000)
    assert _sim(p, c).path == "generic"
    p = Params(nx=16, ny=16, nz=16, bc=(1,) * 6, integrator=2, tmax=1.0, dtoutput=1.0)
    c = problems.random_smooth(p, seed=1, with_vz=True)
    assert _sim(p, c).path == "stage3d"
    assert _sim(dataclasses.replace(p, integrator=1), c).path == "generic"  # Euler: in place


@pytest.mark.parametrize("source", ["none", "gravity", "point"])
def test_stage3d_equals_generic_path_bitwise(monkeypatch, source):
    """The 3D stage (z fluxes + fused x-y stage per plane) uses the generic
    path's expressions: both give the same bits in parity mode.  Without a
    source the last stage also reduces the CFL speed; with constant gravity
    (RK2) or a point mass (RK3) the kick and a separate CFL pass follow it."""
    integ = {"none": 3, "gravity": 2, "point": 3}[source]
    grav = (0.05, -0.1, 0.08) if source == "gravity" else (0.0, 0.0, 0.0)
    p = Params(nx=40, ny=36, nz=32, bc=(1, 3, 1, 1, 2, 1), integrator=integ, grav=grav,
               tmax=1.0, dtoutput=1.0, stepmax=6)
    c = problems.random_smooth(p, seed=8, with_vz=True)
    mass = [(0.5, 0.45, 0.5, 0.55, 0.1)]
    a = _sim(p, c)
    if source == "point":
        a.set_point_gravity(mass)
    monkeypatch.setenv("GK_STAGE3D", "0")  # read whenever the path is chosen
    b = _sim(p, c)
    if source == "point":
        b.set_point_gravity(mass)
    monkeypatch.delenv("GK_STAGE3D")
    assert a.path == "stage3d" and b.path == "generic"
    a.run(p.tmax, p.dtoutput)
    b.run(p.tmax, p.dtoutput)
    assert a.dt_log() == b.dt_log()
    assert np.array_equal(a.download(), b.download())


def test_fast_mode_3d_within_tolerance():
    p = Params(nx=32, ny=32, nz=32, bc=(1,) * 6, integrator=2, tmax=1.0, dtoutput=1.0, stepmax=60)
    c = problems.random_smooth(p, seed=9, with_vz=True)
    ref, ref_dts, _ = _oracle_run(p, c)
    s = _sim(p, c, mode="fast")
    assert s.path == "stage3d"
    s.run(p.tmax, p.dtoutput)
    assert len(s.dt_log()) == 60
    errs = rel_linf(active(p, s.download()), ref)
    assert max(errs) <= FAST_TOL, errs


@pytest.mark.parametrize("n", [256])
def test_fast_mode_within_tolerance_100_steps(n):
    p, c = problems.kh(n)
    p = dataclasses.replace(p, stepmax=100)
    ref, ref_dts, _ = _oracle_run(p, c)
    s = _sim(p, c, mode="fast")
    s.run(p.tmax, p.dtoutput)
    assert len(s.dt_log()) == 100
    errs = rel_linf(active(p, s.download()), ref)
    assert max(errs[v] for v in (0, 1, 2, 4)) <= FAST_TOL, errs


def test_advance_semantics_match_reference_loop():
    """Sim::Advance clamps the last dt to the output time and keeps t, step
    and isContinue across calls (sim.cpp:69-117); stepmax stops the run."""
    p, c = problems.kh(48)
    p = dataclasses.replace(p, tmax=0.05, dtoutput=0.013, stepmax=-1)
    o = gk_oracle.OracleSim(p, c)
    s = _sim(p, c)
    for _ in range(3):
        o_dts = o.advance(0.013)
        t, step, cont = s.advance(0.013)
        assert t == o.time and step == o.step and cont == o.is_continue
    assert s.dt_log()[-len(o_dts):] == o_dts
    q = dataclasses.replace(p, stepmax=7)
    s2 = _sim(q, c)
    t, step, cont = s2.advance(1.0)
    assert step == 7 and not cont
    t2, step2, _ = s2.advance(1.0)
    assert (t2, step2) == (t, step)


def test_nonfinite_state_is_reported():
    """A NaN injected on the host into the uploaded state is reported by the
    CFL reduction as an error, not propagated silently."""
    from gaukuk_b200._lib import GkError
    p, c = problems.kh(32)
    c = c.copy()
    c[0, 2, 10, 10] = np.nan
    with pytest.raises(GkError):
        _sim(p, c)


def test_kh4096_parity_vs_fast_and_conservation():
    """Full size (4096^2): parity and fast modes agree to 1e-12 after a few
    steps and both conserve mass and energy to round-off."""
    p, c = problems.kh(4096)
    s1 = _sim(p, c, "parity")
    s2 = _sim(p, c, "fast")
    assert s1.run_steps(4) == 4 and s2.run_steps(4) == 4
    a, b = active(p, s1.download()), active(p, s2.download())
    errs = rel_linf(b, a)
    assert max(errs[v] for v in (0, 1, 2, 4)) < FAST_TOL, errs
    m0 = active(p, c).sum(axis=(1, 2, 3))
    for x in (a, b):
        m = x.sum(axis=(1, 2, 3))
        assert abs(m[0] - m0[0]) / m0[0] < 1e-13
        assert abs(m[4] - m0[4]) / m0[4] < 1e-13


def test_kh4096_two_steps_against_oracle():
    p, c = problems.kh(4096)
    p = dataclasses.replace(p, stepmax=2)
    ref, ref_dts, _ = _oracle_run(p, c)
    s = _sim(p, c)
    s.run(p.tmax, p.dtoutput)
    assert s.dt_log() == ref_dts
    assert np.array_equal(active(p, s.download()), ref)


def test_fastmath_refinements_within_error_bound():
    """The fast mode's reciprocal / sqrt / rsqrt refinements stay within a few
    ulp of CUDA's IEEE results over [2^-60, 2^60]."""
    import ctypes
    from gaukuk_b200 import _lib
    L = _lib.load()
    w = (ctypes.c_double * 3)()
    _lib.check(L.gk_fastmath_check(1 << 22, 12345, w))
    assert w[0] <= 2.0 and w[1] <= 2.0 and w[2] <= 2.0, list(w)


def _extreme_state(n, with_vz, seed=0, nz=1):
    """A random 2D or 3D state at the edges of the scheme: densities
    log-uniform in [1e-12, 1e2] with 2 % negative (the floor resets them),
    velocities up to 10, pressures log-uniform in [1e-14, 10], and 5 % of the
    cells with negative internal energy (the pressure floor), under mixed
    sides."""
    p = Params(nx=n, ny=n, nz=nz, bc=(1, 3, 2, 0, 3, 1) if nz > 1 else (1, 3, 2, 0, 1, 1),
               integrator=2, tmax=1.0, dtoutput=1.0, stepmax=3)
    rng = np.random.default_rng(seed)
    sh = (nz, n, n) if nz > 1 else (n, n)
    rho = 10 ** rng.uniform(-12, 2, sh)
    rho[rng.random(sh) < 0.02] = -1e-3
    vx, vy = rng.uniform(-10, 10, sh), rng.uniform(-10, 10, sh)
    vz = rng.uniform(-10, 10, sh) if with_vz else np.zeros(sh)
    c = problems.prim_to_cons(p, rho, vx, vy, vz, 10 ** rng.uniform(-14, 1, sh))
    g = p.ng
    a = c[:, g:g + nz, g:g + n, g:g + n] if nz > 1 else c[:, g, g:g + n, g:g + n]
    neg = rng.random(sh) < 0.05
    a[4][neg] = 0.25 * (a[1][neg] ** 2 + a[2][neg] ** 2 + a[3][neg] ** 2) / np.abs(a[0][neg])
    return p, c


@pytest.mark.parametrize("path", ["fused2d", "generic", "stage3d"])
def test_extreme_states_bitwise(path):
    """Every face's reconstruction and Riemann solve, and the floors, on a
    state full of near-vacuum, negative-density and negative-energy cells:
    three steps equal the oracle's bit for bit, dt sequence included, and
    the floors fired.  (At 96^2 the same recipe goes non-finite in the
    oracle too; the device then stops with GK_ERR_NONFINITE.)"""
    p, c = (_extreme_state(16, True, nz=16) if path == "stage3d"
            else _extreme_state(64, path == "generic"))
    ref, ref_dts, _ = _oracle_run(p, c)
    s = _sim(p, c)
    assert s.path == path
    s.run(p.tmax, p.dtoutput)
    assert s.dt_log() == ref_dts and len(ref_dts) == 3
    got = active(p, s.download())
    assert np.isfinite(got).all() and np.array_equal(got, ref)
    den, pre = s.floor_hits()
    assert den > 0 and pre > 0


@pytest.mark.parametrize("state", ["kh", "smooth", "rt"])
def test_fast_face_fluxes_close_to_parity(state):
    """Face by face, the fast mode's reconstruction and HLLC (FMA
    contraction, refined reciprocals and roots, only the selected side, half
    slopes) stay within 1e-13 of parity mode, whose fluxes are the
    reference's bits (scale: the largest |flux| of each component).  The
    extreme states above are left out on purpose: there floored cells carry
    velocities near 1e13, S - v cancels to rounding noise in both modes, and
    the two roundings differ."""
    from gaukuk_b200.learned import face_fluxes
    if state == "kh":
        p, c = problems.kh(192, seed=3)
    elif state == "rt":
        p, c = problems.rt(64, 192)
    else:
        p = Params(nx=160, ny=128, bc=(1,) * 6, integrator=2, tmax=1.0, dtoutput=1.0)
        c = problems.random_smooth(p, seed=5)
    out = {}
    for mode in ("parity", "fast"):
        s = _sim(p, c, mode=mode)
        out[mode] = face_fluxes(s)
        s.close()
    for a, b in zip(out["parity"], out["fast"]):
        assert np.isfinite(a).all() and np.isfinite(b).all()
        for v in range(4):
            scale = np.abs(a[v]).max()
            assert np.abs(b[v] - a[v]).max() <= 1e-13 * scale, (v, np.abs(b[v] - a[v]).max() / scale)
