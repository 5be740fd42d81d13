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


def test_zero_model_is_plain_hllc_bitwise():
    from gaukuk_b200.sim import Sim
    p, c = problems.kh(96, ny=80, seed=1)
    blob = np.zeros(learned.NMODEL, dtype=np.float32)
    blob[learned.NPARAM + 16:learned.NPARAM + 32] = 1.0  # input deviations
    blob[learned.NPARAM + 36:] = 1.0                    # output deviations
    a, b = Sim(p, c, mode="parity"), Sim(p, c, mode="parity")
    learned.install(b, blob)
    assert b.path == "generic"
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
