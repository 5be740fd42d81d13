"""Host-side pieces of the learned flux correction and its CPU oracle."""
import numpy as np
import pytest

from gaukuk_b200 import learned, problems

mlp_oracle = pytest.importorskip("mlp_oracle")


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(48, 16))
    T = rng.normal(size=(48, 4)) * 0.1
    blob = learned.init_model(X, T, seed=1)[:learned.NPARAM].astype(np.float64)
    _, g, _ = mlp_oracle.forward_backward(blob, X, T, rounding=False)
    eps = 1e-6
    for i in (0, 100, 1030, 1100, 5000, 5250, 5505):
        bp, bm = blob.copy(), blob.copy()
        bp[i] += eps
        bm[i] -= eps
        fd = (mlp_oracle.forward_backward(bp, X, T, False)[0]
              - mlp_oracle.forward_backward(bm, X, T, False)[0]) / (2 * eps) / len(X)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_pair_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(4)
    X, T = rng.normal(size=(16, 16)), rng.normal(size=(16, 4))
    b = learned.init_model(X, T, seed=2)[:learned.NPARAM].astype(np.float64)
    b[-4 - 4 * 64:] = rng.normal(size=4 + 4 * 64) * 0.3  # a last layer of some size
    for w in (0.0, 0.7, 1.0):
        _, g, _ = mlp_oracle.forward_backward(b, X, T, False, pair_w=w)
        for i in rng.choice(len(b), 12, replace=False):
            eps = 1e-6
            bp, bm = b.copy(), b.copy()
            bp[i] += eps
            bm[i] -= eps
            fd = (mlp_oracle.forward_backward(bp, X, T, False, pair_w=w)[0]
                  - mlp_oracle.forward_backward(bm, X, T, False, pair_w=w)[0]) / (2 * eps) / len(X)
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (w, i, fd, g[i])
    # w = 0 is the per-sample squared error
    assert np.isclose(mlp_oracle.forward_backward(b, X, T, False, pair_w=0.0)[0],
                      mlp_oracle.forward_backward(b, X, T, False)[0])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.0078125, 3.14159265, -2.5e-3])
    r = mlp_oracle.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125  # tie to even, exact
    assert abs(r[3] - 3.140625) < 1e-12 and np.all(np.abs(r - x) <= 2 ** -8 * np.abs(x))


def test_features_of_a_uniform_state():
    p, c = problems.kh(16, amp=0.0, noise=0.0, rho_in=1.0, rho_out=1.0)
    a = learned.active2d(p, c)
    for d in (0, 1):
        X, S = learned.face_features(p, a, d)
        cs = np.sqrt(1.4 * 2.5 / 1.0)
        assert np.allclose(X[:, 0::4], 0) and np.allclose(X[:, 3::4], 0)
        v = 0.5 / cs if d == 0 else 0.0
        assert np.allclose(np.abs(X[:, 1]), v)
        assert np.allclose(S[:, 0], cs)


def test_restriction_is_conservative():
    p, c = problems.kh(32, seed=3)
    q, r = learned.restrict(p, c, 4)
    assert q.nx == 8 and r.shape == q.shape
    for v in range(5):
        assert np.isclose(learned.active2d(q, r)[v].sum() * 16, learned.active2d(p, c)[v].sum())


def test_model_blob_layout():
    X = np.random.default_rng(1).normal(size=(100, 16))
    Y = np.random.default_rng(2).normal(size=(100, 4))
    b = learned.init_model(X, Y)
    assert b.size == learned.NMODEL == 5548 and b.dtype == np.float32
    Xn, Yn = learned.standardise(b, X, Y)
    assert np.allclose(Xn.mean(0), 0, atol=1e-5) and np.allclose(Yn.std(0), 1, atol=1e-3)


def test_hll_dissipation_vanishes_on_a_uniform_state_and_not_at_a_jump():
    """(1/2) max(|vn| + c) |U_R - U_L| at each face: zero where the PLM face
    states agree, positive across the shear layers of a KH state, and the
    same face count as the features."""
    p, c = problems.kh(16, amp=0.0, noise=0.0)
    a = learned.active2d(p, c)
    uniform = np.broadcast_to(a[:, :1, :1], a.shape).copy()
    for d in (0, 1):
        D = learned.hll_dissipation(p, uniform, d)
        assert D.shape == (16 * 16, 4) and np.all(D == 0.0)
    Dy = learned.hll_dissipation(p, a, 1)
    assert np.all(Dy >= 0.0) and Dy[:, 0].max() > 0.0
    assert Dy.shape[0] == learned.face_features(p, a, 1)[0].shape[0]
    # x faces see no jump: density and vx change only along y
    assert np.all(learned.hll_dissipation(p, a, 0) == 0.0)


def test_stencil_variation_and_face_rotation():
    X = np.zeros((2, 16))
    X[1, 4:8] = [1.0, -2.0, 0.5, 0.0]  # the second cell differs from its two neighbours
    assert learned.stencil_variation(X).tolist() == [0.0, 2 * 3.5]
    planes = np.arange(4 * 6, dtype=np.float64).reshape(4, 2, 3)
    x = learned.rotate_to_face(planes, 0)
    y = learned.rotate_to_face(planes, 1)
    assert np.array_equal(x[:, 1], planes[1].ravel()) and np.array_equal(x[:, 2], planes[2].ravel())
    assert np.array_equal(y[:, 1], planes[2].ravel()) and np.array_equal(y[:, 2], planes[1].ravel())
    assert np.array_equal(x[:, [0, 3]], y[:, [0, 3]])


def test_summary_leaves_out_diverged_runs():
    def run(l1, secs, diverged=False):
        return {"l1_at_64": l1, "seconds": secs, "diverged": diverged}

    rows = [{"plain_64": run([1.0, 2.0], 1.0), "plain_128": run([0.5, 1.0], 4.0),
             "learned_64": run([0.8, 1.5], 2.0)},
            {"plain_64": run([3.0, 4.0], 3.0), "plain_128": run([1.5, 2.0], 8.0),
             "learned_64": run([9.0, 9.0], 9.0, diverged=True)}]
    s = learned.summarise(rows, 64)
    assert s["plain_64"]["mean_l1_at_64"] == [2.0, 3.0] and s["plain_64"]["mean_seconds"] == 2.0
    assert s["plain_128"]["median_l1_at_64"] == [1.0, 1.5]
    assert s["learned_64"]["runs"] == 1 and s["learned_64"]["diverged"] == 1
    assert s["learned_64"]["mean_l1_at_64"] == [0.8, 1.5] and s["learned_64"]["mean_seconds"] == 2.0
