"""The learned field's oracle (oracle/mvc_field.py) checked on the CPU: with
the bf16 rounding switched off, its backward pass matches central
differences of its loss, its Jacobian matches central differences of its
position, and the folded output layer equals sum_j w_j v_j."""
import numpy as np
import pytest

from oracle import mvc_field as of


@pytest.fixture
def exact(monkeypatch):
    monkeypatch.setattr(of, "bf16", lambda a: np.asarray(a, np.float64))
    monkeypatch.setattr(of, "EMULATE_F32", False)


def small_net(V, seed):
    rng = np.random.default_rng(seed)
    P = {"W1": rng.normal(0, np.sqrt(2 / 64), (128, 64))}
    for l in (2, 3, 4):
        P[f"W{l}"] = rng.normal(0, np.sqrt(2 / 128), (128, 128))
    for l in (1, 2, 3, 4):
        P[f"b{l}"] = rng.normal(0, 0.1, 128)
    P["W5"] = rng.normal(0, 0.05, (V, 128))
    P["b5"] = 1.0 / V + rng.normal(0, 1e-2, V)
    return P


def setup(V=12, n=16, seed=0):
    rng = np.random.default_rng(seed)
    verts = rng.normal(size=(V, 3))
    x = rng.uniform(-0.8, 0.8, (n, 3))
    wt = rng.dirichlet(np.ones(V), n)
    enc = np.array([0.05, -0.1, 0.02, 1.0 / 1.3])
    return small_net(V, seed + 1), x, wt, verts, enc


def total_loss(P, x, wt, verts, enc, lam):
    (lw, lr), _ = of.loss_and_grads(P, x, wt, verts, enc, lam)
    return lw + lam * lr


def test_backward_matches_central_differences(exact):
    P, x, wt, verts, enc = setup()
    lam = 0.7
    _, g = of.loss_and_grads(P, x, wt, verts, enc, lam)
    rng = np.random.default_rng(3)
    for k in of.NAMES:
        for _ in range(4):
            idx = tuple(rng.integers(0, d) for d in P[k].shape)
            h = 1e-5
            old = P[k][idx]
            P[k][idx] = old + h
            lp = total_loss(P, x, wt, verts, enc, lam)
            P[k][idx] = old - h
            lm = total_loss(P, x, wt, verts, enc, lam)
            P[k][idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[k][idx]) <= 1e-6 + 1e-4 * abs(fd), (k, idx, fd, g[k][idx])


@pytest.mark.parametrize("which", ["deformed", "raw"])
def test_jacobian_and_folded_output(exact, monkeypatch, which):
    P, x, _, rest, enc = setup(V=20, n=8, seed=4)
    rng = np.random.default_rng(5)
    cur = rest + 0.1 * rng.normal(size=rest.shape) if which == "deformed" else None
    # float64 M so that linear precision holds to rounding
    Vb = np.concatenate([np.ones((1, len(rest))), rest.T], 0)
    monkeypatch.setattr(of, "lp_matrix", lambda v: np.linalg.inv(Vb @ Vb.T))
    pos, F = of.position_and_jacobian(P, x, cur, enc, rest)
    w0 = of.pou(of.forward(P, x, enc)[0])
    w = of.weights(P, x, enc, rest)
    if cur is None:
        np.testing.assert_allclose(pos, w0 @ rest, atol=1e-12)
    else:
        np.testing.assert_allclose(pos, w @ cur, atol=1e-12)
    np.testing.assert_allclose(w.sum(1), 1.0, atol=1e-12)
    np.testing.assert_allclose(w @ rest, x, atol=1e-12)  # linear precision
    h = 1e-6
    for k in range(3):
        d = np.zeros(3)
        d[k] = h
        pp, _ = of.position_and_jacobian(P, x + d, cur, enc, rest)
        pm, _ = of.position_and_jacobian(P, x - d, cur, enc, rest)
        np.testing.assert_allclose(F[:, :, k], (pp - pm) / (2 * h), atol=1e-6, rtol=1e-6)


def test_affine_cage_motion_is_exact(exact, monkeypatch):
    """With the projection, an affine motion of the cage moves every point
    affinely, whatever the network."""
    P, x, _, rest, enc = setup(V=20, n=8, seed=6)
    Vb = np.concatenate([np.ones((1, len(rest))), rest.T], 0)
    monkeypatch.setattr(of, "lp_matrix", lambda v: np.linalg.inv(Vb @ Vb.T))
    A = np.array([[1.1, 0.2, -0.1], [0.05, 0.9, 0.3], [-0.2, 0.1, 1.2]])
    t = np.array([0.3, -0.2, 0.5])
    pos, F = of.position_and_jacobian(P, x, rest @ A.T + t, enc, rest)
    np.testing.assert_allclose(pos, x @ A.T + t, atol=1e-10)
    np.testing.assert_allclose(F, np.broadcast_to(A, F.shape), atol=1e-9)


def test_bf16_rounding():
    # bf16 keeps 7 fraction bits: ulp(1) = 2^-7, ties at odd multiples of 2^-8
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9,
                  -3.14159], np.float32)
    r = of.bf16(v)
    np.testing.assert_array_equal(r[:5], [1.0, 1.0, 1.015625, 1.0078125, 1.0])
    assert r[5] == -3.140625
