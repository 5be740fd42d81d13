"""The learned flux correction on the GPU: training kernels against the CPU
oracle, the flux tap's conservation identity, and the corrected solver's
fall-back and conservation properties."""
import dataclasses

import numpy as np
import pytest

from gaukuk_b200 import learned, problems
from helpers import active

pytestmark = pytest.mark.gpu
mlp_oracle = pytest.importorskip("mlp_oracle")


def _data(n=2048, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 16))
    a = rng.normal(size=(16, 4))
    Y = np.tanh(X @ a * 0.3) + 0.05 * rng.normal(size=(n, 4))
    return X.astype(np.float32), Y.astype(np.float32)


def test_gradient_matches_cpu_oracle():
    X, Y = _data(1024)
    blob = learned.init_model(X, Y, seed=3)
    tr = learned.Trainer(blob, X, Y)
    g, loss = tr.gradient(1024)
    Xn, Yn = learned.standardise(blob, X, Y)
    l_ref, g_ref, _ = mlp_oracle.forward_backward(blob[:learned.NPARAM], Xn, Yn, rounding=True)
    assert abs(loss - l_ref) <= 1e-3 * l_ref
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert err < 1e-2, err
    # and per block (W1, b1, W2, b2, W3, b3)
    cuts = np.cumsum([0, 1024, 64, 4096, 64, 256, 4])
    for a, b in zip(cuts[:-1], cuts[1:]):
        e = np.linalg.norm(g[a:b] - g_ref[a:b]) / (np.linalg.norm(g_ref[a:b]) + 1e-30)
        assert e < 3e-2, (a, b, e)
    tr.close()


def test_pair_loss_gradient_matches_cpu_oracle():
    X, Y = _data(1024, seed=5)
    blob = learned.init_model(X, Y, seed=6)
    tr = learned.Trainer(blob, X, Y)
    tr.set_pair_loss(0.8)
    g, loss = tr.gradient(1024)
    Xn, Yn = learned.standardise(blob, X, Y)
    l_ref, g_ref, _ = mlp_oracle.forward_backward(blob[:learned.NPARAM], Xn, Yn, rounding=True,
                                                  pair_w=0.8)
    assert abs(loss - l_ref) <= 1e-3 * l_ref
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert err < 1e-2, err
    l0 = tr.train(1, batch=1024, lr=1e-3)
    l1 = tr.train(300, batch=1024, lr=3e-3)
    assert l1 < 0.5 * l0, (l0, l1)
    tr.close()


def test_forward_matches_cpu_oracle():
    X, Y = _data(512, seed=1)
    blob = learned.init_model(X, Y, seed=4)
    tr = learned.Trainer(blob, X, Y)
    y = tr.forward()
    Xn, Yn = learned.standardise(blob, X, Y)
    _, _, y_ref = mlp_oracle.forward_backward(blob[:learned.NPARAM], Xn, Yn, rounding=True)
    assert np.max(np.abs(y - y_ref)) < 1e-3 * (1 + np.max(np.abs(y_ref)))
    tr.close()


def test_training_reduces_loss():
    X, Y = _data(8192, seed=2)
    blob = learned.init_model(X, Y, seed=5)
    tr = learned.Trainer(blob, X, Y)
    l0 = tr.train(1, batch=1024, lr=1e-3)
    l1 = tr.train(600, batch=1024, lr=3e-3)
    assert l1 < 0.2 * l0, (l0, l1)
    tr.close()


def test_flux_tap_is_the_restricted_update():
    """The fine run's update restricted to the coarse grid equals the coarse
    flux divergence of the tapped fluxes (RK2 is u - dt/2 (dF(u) + dF(u*)))."""
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(128, seed=4)
    s = Sim(p, c, mode="parity")
    s.run_steps(3)
    r = 4
    q, u0 = learned.restrict(p, s.download(), r)
    nsub, dt = 4, 2e-4
    fx, fy = learned.tap(s, nsub, dt, r)
    _, u1 = learned.restrict(p, s.download(), r)
    a0, a1 = learned.active2d(q, u0), learned.active2d(q, u1)
    T = nsub * dt
    dx, dy = 1.0 / q.nx, 1.0 / q.ny
    for v, pl in ((0, 0), (1, 1), (2, 2), (4, 3)):
        div = (np.roll(fx[pl], -1, axis=1) - fx[pl]) / dx + (np.roll(fy[pl], -1, axis=0) - fy[pl]) / dy
        pred = a0[v] - T * div
        err = np.max(np.abs(pred - a1[v])) / np.max(np.abs(a1[v]))
        assert err < 1e-12, (v, err)
    assert len(s.dt_log()) == 3 and abs(s.get_time() - (sum(s.dt_log()) + T)) < 1e-12


def test_device_correction_matches_the_oracle():
    """k_flux_correct's correction of each face flux equals the CPU oracle's
    forward pass on the Python features, de-standardised, scaled by the flux
    scales and clipped to diss_frac times the HLL dissipation; faces whose
    stencil variation is below tv_min uncorrected."""
    from gaukuk_b200.sim import Sim
    p, c, _ = learned.kh_instance(11, 64, 1.0)
    s = Sim(p, c, mode="fast")
    s.run_steps(20)
    a = learned.active2d(p, s.download())
    fx0, fy0 = learned.face_fluxes(s)
    n = learned.NPARAM
    feats = {d: learned.face_features(p, a, d) for d in (0, 1)}
    # a gate in the widest gap between the middle faces' variations, so both
    # kinds of face occur and none lies near it (the device sums in FP32)
    gs = np.sort(np.concatenate([learned.stencil_variation(feats[d][0]) for d in (0, 1)]))
    lo, hi = len(gs) // 4, 3 * len(gs) // 4
    k = lo + int(np.argmax(np.diff(gs[lo:hi])))
    tv_min = float(0.5 * (gs[k] + gs[k + 1]))
    assert gs[k + 1] - gs[k] > 1e-4 * tv_min
    diss_frac = 0.5
    X, Y = _data(256)
    blob = learned.init_model(X, Y, seed=8)
    blob[n + 32:n + 36] = 0.0

    def raw(d):
        Xf, S = feats[d]
        _, _, yn = mlp_oracle.forward_backward(blob[:n], learned.standardise(blob, Xf),
                                               np.zeros((len(Xf), 4)), rounding=True)
        return np.clip(yn, -4, 4) * np.stack([S[:, 0], S[:, 1], S[:, 1], S[:, 2]], axis=1)

    # output deviations that put about half of the gated corrections above the bound
    ratio = np.concatenate([(diss_frac * learned.hll_dissipation(p, a, d) / np.maximum(np.abs(raw(d)), 1e-300))
                            [learned.stencil_variation(feats[d][0]) >= tv_min] for d in (0, 1)])
    blob[n + 36:n + 40] = np.median(ratio, axis=0)
    learned.install(s, blob, shock_jump=10.0, pos_frac=1.0, tv_min=tv_min, diss_frac=diss_frac)
    fx1, fy1 = learned.face_fluxes(s)
    for d, dF in ((0, (fx1 - fx0)[:, :, :p.nx]), (1, (fy1 - fy0)[:, :p.ny, :])):
        gated = learned.stencil_variation(feats[d][0]) >= tv_min
        ref = raw(d) * blob[n + 36:n + 40] * gated[:, None]
        bound = diss_frac * learned.hll_dissipation(p, a, d)
        clipped = np.abs(ref) > bound
        assert clipped[gated].any() and (~clipped[gated]).any()
        ref = np.clip(ref, -bound, bound)
        got = learned.rotate_to_face(dF, d)
        assert np.all(got[~gated] == 0)
        for o in range(4):
            err = np.linalg.norm(got[:, o] - ref[:, o]) / np.linalg.norm(ref[:, o])
            assert err < 2e-2, (d, o, err)
    s.close()


def test_zero_dissipation_bound_is_plain_hllc():
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(64, seed=5)
    X, Y = _data(256)
    blob = learned.init_model(X, Y, seed=9)
    a, b = Sim(p, c, mode="parity"), Sim(p, c, mode="parity")
    learned.install(b, blob, shock_jump=10.0, pos_frac=1.0, tv_min=0.0, diss_frac=0.0)
    a.run_steps(6)
    b.run_steps(6)
    assert np.array_equal(active(p, a.download()), active(p, b.download()))


@pytest.mark.parametrize("fused", [True, False])
def test_zero_model_is_plain_hllc_bitwise(fused):
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(96, ny=80, seed=1)
    blob = np.zeros(learned.NMODEL, dtype=np.float32)
    blob[learned.NPARAM + 16:learned.NPARAM + 32] = 1.0  # input deviations
    blob[learned.NPARAM + 36:] = 1.0                    # output deviations
    a, b = Sim(p, c, mode="parity"), Sim(p, c, mode="parity")
    learned.install(b, blob, fused=fused)
    assert b.path == ("fused2d" if fused else "generic")
    a.run_steps(12)
    b.run_steps(12)
    assert a.dt_log() == b.dt_log()
    assert np.array_equal(active(p, a.download()), active(p, b.download()))


def test_detector_fallback_is_plain_hllc():
    """With pos_frac = 0, no smoothness gate and no clip every correction
    trips the positivity detector, so the corrected solver must reproduce
    plain HLLC exactly."""
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(64, seed=2)
    X, Y = _data(256)
    blob = learned.init_model(X, Y, seed=6)
    a, b = Sim(p, c, mode="parity"), Sim(p, c, mode="parity")
    learned.install(b, blob, shock_jump=0.5, pos_frac=0.0, tv_min=0.0, diss_frac=-1.0)
    a.run_steps(6)
    b.run_steps(6)
    assert np.array_equal(active(p, a.download()), active(p, b.download()))
    assert learned.detector_count(b) == 6 * 2 * 2 * 64 * 65


def test_corrected_run_conserves_mass_and_changes_the_solution():
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(128, seed=3)
    X, Y = _data(256)
    blob = learned.init_model(X, Y, seed=7)
    blob[learned.NPARAM + 36:] *= 1e-4  # small corrections
    a, b = Sim(p, c, mode="fast"), Sim(p, c, mode="fast")
    learned.install(b, blob, shock_jump=0.5, pos_frac=0.5)
    a.run_steps(20)
    b.run_steps(20)
    ma, mb = active(p, a.download()), active(p, b.download())
    m0 = active(p, c)[0].sum()
    assert abs(mb[0].sum() - m0) / m0 < 1e-13
    assert abs(mb[4].sum() - active(p, c)[4].sum()) / active(p, c)[4].sum() < 1e-13
    assert not np.array_equal(ma, mb)


def test_trained_correction_against_plain_on_a_held_out_case():
    """What the trained network gains: data from ensemble-run fine grids
    (4 training seeds, 256^2 restricted to 64^2), 3000 Adam steps on the
    device, then one held-out seed at 64^2 to t = 0.5 against plain 64^2 and
    plain 128^2, L1 density error against the 256^2 plain run.  The printed
    line states the outcome.  Asserted: the learned run finishes, conserves
    mass, and -- the measured result at every configuration tried -- does
    not reach the accuracy of plain 128^2."""
    X, Y = learned.generate([1000, 1001, 1002, 1003], coarse=64, t_end=0.5, snapshots=4,
                            frac=0.5, noise=0.03, log=None)
    blob = learned.init_model(X, Y, seed=0)
    tr = learned.Trainer(blob, X, Y)
    first = tr.train(1, batch=8192, lr=1e-3)
    last = tr.train(3000, batch=8192, lr=1e-3, seed=1)
    model = tr.model()
    tr.close()
    assert last < first
    ev = learned.evaluate(model, [5000], coarse=64, t_end=0.5, times=(0.25, 0.5), log=None)
    run = ev["runs"][0]
    plain, plain2, lrn = run["plain_64"], run["plain_128"], run["learned_64"]
    print(f"\nheld-out seed 5000, L1(rho) at t = 0.25, 0.5 against 256^2: plain 64^2 "
          f"{plain['l1_at_64']}, plain 128^2 {plain2['l1_at_64']}, learned 64^2 {lrn['l1_at_64']} "
          f"(diverged: {lrn['diverged']}); learned / plain at t = 0.5: "
          f"{lrn['l1_at_64'][-1] / plain['l1_at_64'][-1]:.3g}")
    assert not lrn["diverged"]
    assert np.isfinite(lrn["l1_at_64"]).all()
    assert lrn["mass_drift"] < 1e-13
    assert lrn["l1_at_64"][-1] > plain2["l1_at_64"][-1]


# Gates for the model below (outputs scaled by 0.05): at the initial states
# the positivity ratio max(|c_mass| dt/dx / rho_min, |c_energy| dt/dx / e_min)
# is about 0.0065 in the dense layer and 0.0093 outside it for KH, 0.008 to
# 0.0117 for RT, and the stencil variation's median is about 0.0012, so each
# gate splits the faces: corrected, vetoed, smooth (and clipped, RT's
# pressure jumps above 0.1 % vetoed as shocks).
GATE_KH = dict(shock_jump=0.5, pos_frac=0.008, tv_min=0.0012, diss_frac=-1.0)
GATE_CLIP = dict(shock_jump=0.5, pos_frac=0.008, tv_min=0.0012, diss_frac=0.5)
GATE_RT = dict(shock_jump=0.001, pos_frac=0.01, tv_min=0.0012, diss_frac=0.5)


def _fused_case(name):
    """(params, state, tiling or None, gate, vetoes expected) of the
    fused-correction cases."""
    from gaukuk_b200.config import BC_PERIODIC, BC_REFLECTIVE
    if name == "kh_rk2":
        p, c = problems.kh(96, ny=80, seed=12)
        return p, c, None, GATE_KH, True
    if name == "kh_rk3_tiles128_clip":
        p, c = problems.kh(150, ny=70, seed=13)
        return dataclasses.replace(p, integrator=3), c, (128, 4), GATE_CLIP, False
    if name == "rt_rk3_gravity_tiles64":
        p, c = problems.rt(64, 192)
        assert p.integrator == 3 and p.bc[2] == BC_REFLECTIVE and p.bc[0] == BC_PERIODIC
        return p, c, (64, 5), GATE_RT, True
    if name == "kh_first_order":
        p, c = problems.kh(64, seed=14)
        return dataclasses.replace(p, rc_order=1), c, None, GATE_KH, True
    raise KeyError(name)


def _model():
    X, Y = _data(256)
    blob = learned.init_model(X, Y, seed=21)
    blob[learned.NPARAM + 36:] *= 0.05
    return blob


# A gate that decides nothing: no shocks, no positivity vetoes, no smooth
# faces, no clip.
GATE_OPEN = dict(shock_jump=1e30, pos_frac=1e30, tv_min=0.0, diss_frac=-1.0)


def _pair(name, mode, blob, gate=None):
    from gaukuk_b200.sim import Sim
    p, c, tiling, case_gate, _ = _fused_case(name)
    gate = case_gate if gate is None else gate
    a, b = Sim(p, c, mode=mode), Sim(p, c, mode=mode)
    for s in (a, b):
        if tiling:
            s.set_tiling(*tiling)
    learned.install(a, blob, fused=True, **gate)
    learned.install(b, blob, fused=False, **gate)
    assert a.path == "fused2d" and b.path == "generic"
    return p, c, a, b


CASES = ["kh_rk2", "kh_rk3_tiles128_clip", "rt_rk3_gravity_tiles64", "kh_first_order"]


@pytest.mark.parametrize("case", CASES)
def test_fused_correction_is_the_correction_pass_bitwise(case):
    """Parity mode: the fused 2D stage with the network at every face (the
    default) gives the generic path's correction pass bit for bit -- state,
    dt sequence and detector count -- across strip and segment boundaries
    (small tiles, both CTA widths), RK2 and RK3, gravity, reflective sides
    and first order.  The gate settings make every branch occur: corrected,
    clipped, vetoed (shock and positivity) and smooth faces."""
    from gaukuk_b200.sim import Sim
    p, c, a, b = _pair(case, "parity", _model())
    a.run_steps(8)
    b.run_steps(8)
    assert a.dt_log() == b.dt_log()
    assert np.array_equal(active(p, a.download()), active(p, b.download()))
    na, nb = learned.detector_count(a), learned.detector_count(b)
    assert na == nb
    plain = Sim(p, c, mode="parity")
    plain.run_steps(8)
    faces = 8 * (3 if p.integrator == 3 else 2) * (p.ny * (p.nx + 1) + p.nx * (p.ny + 1))
    print(f"\n{case}: {na} of {faces} faces vetoed")
    assert na < faces
    assert na > 0 or not _fused_case(case)[4]
    assert not np.array_equal(active(p, a.download()), active(p, plain.download()))
    for s in (a, b, plain):
        s.close()


@pytest.mark.parametrize("case", ["kh_rk2", "rt_rk3_gravity_tiles64"])
def test_fused_correction_close_to_the_correction_pass_in_fast_mode(case):
    """Fast mode: the fused stage and the generic path round their fluxes
    differently in the last bits, and so do the network's inputs.  With a
    gate that makes no threshold decision (a last-bit difference could flip
    a face across tv_min or a veto, which parity mode's bitwise tests cover)
    the two stay within the fast-mode tolerance (1e-12 relative; momentum
    components against the momentum's magnitude, as RT's x-momentum starts
    at exactly zero) after 8 steps."""
    p, c, a, b = _pair(case, "fast", _model(), gate=GATE_OPEN)
    a.run_steps(8)
    b.run_steps(8)
    ga, gb = active(p, a.download()), active(p, b.download())
    mscale = max(float(np.max(np.abs(gb[1]))), float(np.max(np.abs(gb[2]))))
    scale = {0: np.max(np.abs(gb[0])), 1: mscale, 2: mscale, 4: np.max(np.abs(gb[4]))}
    err = max(float(np.max(np.abs(ga[v] - gb[v])) / scale[v]) for v in (0, 1, 2, 4))
    dev = max(abs(x - y) / y for x, y in zip(a.dt_log(), b.dt_log()))
    print(f"\n{case} fast: fused vs pass rel Linf {err:.2e}, dt {dev:.2e}, vetoed "
          f"{learned.detector_count(a)} / {learned.detector_count(b)}")
    assert err <= 1e-12 and dev <= 1e-12
    assert learned.detector_count(a) == learned.detector_count(b) == 0
