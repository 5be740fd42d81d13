"""Physics checks of the configurations on the GPU path: Sod against the
exact Riemann solution, Rayleigh-Taylor's mirror symmetry, and the full
Kelvin-Helmholtz 256^2 run to t = 2 conserving mass and energy."""
import numpy as np
import pytest

from gaukuk_b200 import problems
from helpers import active

pytestmark = pytest.mark.gpu
rx = pytest.importorskip("riemann_exact")
gk_oracle = pytest.importorskip("gk_oracle")

SOD_L, SOD_R = (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)


def _sod_l1(p, cons, t):
    n = p.nx
    a = cons[:, p.ng, p.ng, p.ng:p.ng + n]
    xl = np.arange(n) / n
    rho, m, e = rx.cell_average(xl, xl + 1.0 / n, t, 0.5, SOD_L, SOD_R)
    return np.abs(a[0] - rho).mean(), np.abs(a[1] - m).mean(), np.abs(a[4] - e).mean()


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_sod_against_the_exact_solution(mode):
    """The Sod configuration (256 cells, PLM + HLLC + RK2, CFL 0.4, outflow,
    t = 0.2) on the GPU: its L1 errors against the exact cell averages equal
    the oracle's (parity mode bit for bit, fast mode to 1e-12) and are small."""
    from gaukuk_b200.sim import Sim
    p, c = problems.sod(256)
    o = gk_oracle.OracleSim(p, c)
    o.run(0.2, 0.2)
    ref = _sod_l1(p, o.get_cons(), o.time)
    with Sim(p, c, mode=mode) as s:
        s.run(0.2, 0.2)
        assert s.get_step() == o.step == 280
        got = _sod_l1(p, s.download(), s.get_time())
        m = active(p, s.download())[0].sum() / 256
    assert m == pytest.approx(0.5625, abs=1e-14)
    assert ref[0] < 2.5e-3
    for a, b in zip(got, ref):
        assert (a == b) if mode == "parity" else abs(a - b) <= 1e-12 * max(b, 1e-300)


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_rayleigh_taylor_stays_mirror_symmetric(mode):
    """The RT initial state is even in x (rho, p, vy) with vx = 0, so the
    solution must stay mirror-symmetric: rho, vy, E even and x-momentum odd.
    Parity mode keeps it bit for bit (as the oracle does); fast mode, whose
    contracted FMAs need not be mirror-exact, to 1e-10 after 300 steps."""
    from gaukuk_b200.sim import Sim
    p, c = problems.rt(64, 192)
    with Sim(p, c, mode=mode) as s:
        s.run_steps(300)
        a = active(p, s.download())
    tol = 0.0 if mode == "parity" else 1e-10
    for v, sign in ((0, 1), (1, -1), (2, 1), (4, 1)):
        d = np.abs(a[v] - sign * a[v][..., ::-1]).max() / np.abs(a[v]).max()
        assert d <= tol, (v, d)
    assert np.abs(a[1]).max() > 1e-6  # the instability has started to move fluid sideways


def test_kh256_to_t2_conserves():
    """The KH 256^2 configuration run to t = 2 (fast mode): periodic, so mass,
    momentum and total energy are conserved to round-off."""
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(256)
    a0 = active(p, c)
    with Sim(p, c, mode="fast") as s:
        s.run(2.0, 2.0)
        assert abs(s.get_time() - 2.0) < 1e-12
        a = active(p, s.download())
    for v in (0, 4):
        assert abs(a[v].sum() - a0[v].sum()) / a0[v].sum() < 1e-12, v
    for v in (1, 2):
        assert abs(a[v].sum() - a0[v].sum()) / a0[0].sum() < 1e-12, v


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_floor_repairs_are_counted(mode):
    """Two streams rushing apart with a pressure (1e-20) below the floor
    (1e-16): every stage repairs the cells whose pressure stays below it (the
    reference does so silently) and gk_floor_hits counts them; the parity run
    still equals the oracle bit for bit.  A smooth KH run repairs nothing."""
    from gaukuk_b200.sim import Sim
    p, _ = problems.sod(128)
    x = (np.arange(p.nx) + 0.5) / p.nx
    z = np.zeros(p.nx)
    c = problems.prim_to_cons(p, np.ones(p.nx), np.where(x < 0.5, -3.0, 3.0), z, z,
                              np.full(p.nx, 1e-20))
    with Sim(p, c, mode=mode) as s:
        s.run(0.02, 0.02)
        den, pre = s.floor_hits()
        got = s.download()
    assert den + pre > 0 and np.isfinite(got).all()
    if mode == "parity":
        o = gk_oracle.OracleSim(p, c)
        o.run(0.02, 0.02)
        assert np.array_equal(active(p, got), active(p, o.get_cons()))
    pk, ck = problems.kh(64)
    with Sim(pk, ck, mode=mode) as s:
        s.run_steps(20)
        assert s.floor_hits() == (0, 0)
