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
