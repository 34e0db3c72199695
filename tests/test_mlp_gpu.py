"""Surrogate network training kernels (FP32 forward, backward, Adam) against the FP64 NumPy
oracle of the same network."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import mlp_oracle as mo  # noqa: E402
from tiger_nga_b200 import capi  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chem():
    return capi.FiniteChem("grimech30", "fp64")


def data(rows, n_in, n_out, in_pad, out_pad, seed=0):
    rng = np.random.default_rng(seed)
    X = np.zeros((rows, in_pad), np.float32)
    X[:, :n_in] = rng.normal(size=(rows, n_in))
    T = np.zeros((rows, out_pad), np.float32)
    T[:, :n_out] = rng.normal(size=(rows, n_out))
    w = np.zeros(out_pad, np.float32)
    w[:n_out] = rng.uniform(0.5, 2.0, n_out)
    return X, T, w


def to64(params):
    return [(W.astype(np.float64), b.astype(np.float64)) for W, b in params]


def test_forward_and_gradients_match_fp64_oracle(chem):
    net = capi.Mlp(chem, 38, 37, hidden=256, layers=4, seed=3)
    X, T, w = data(512, 38, 37, net.in_pad, net.out_pad)
    p = to64(net.get())
    Y = net.forward(X).cpu().numpy()
    Yo, _ = mo.forward(p, X.astype(np.float64))
    assert np.max(np.abs(Y - Yo)) / np.max(np.abs(Yo)) < 1e-5
    loss, g = net.grad(X, T, w)
    lo, go = mo.loss_and_grads(p, X.astype(np.float64), T.astype(np.float64), w.astype(np.float64), n_out=37)
    assert abs(loss - lo) / lo < 1e-5
    for (gW, gb), (oW, ob) in zip(g, go):
        assert np.max(np.abs(gW - oW)) <= 1e-4 * np.max(np.abs(oW)) + 1e-12
        assert np.max(np.abs(gb - ob)) <= 1e-4 * np.max(np.abs(ob)) + 1e-12
    # the zero padding of inputs/outputs carries no gradient
    assert np.all(g[0][0][:, 38:] == 0.0) and np.all(g[-1][0][37:, :] == 0.0)


def test_asymmetric_loss_gradients_match_fp64_oracle(chem):
    """The error gate's loss: squared errors of outputs below their target weigh 4x."""
    net = capi.Mlp(chem, 20, 2, hidden=64, layers=2, seed=5)
    net.set_under_weight(4.0)
    X, T, w = data(384, 20, 2, net.in_pad, net.out_pad, seed=6)
    p = to64(net.get())
    loss, g = net.grad(X, T, w)
    lo, go = mo.loss_and_grads(p, X.astype(np.float64), T.astype(np.float64), w.astype(np.float64), n_out=2,
                               under=4.0)
    l1, _ = mo.loss_and_grads(p, X.astype(np.float64), T.astype(np.float64), w.astype(np.float64), n_out=2)
    assert abs(loss - lo) / lo < 1e-5 and abs(lo - l1) / l1 > 0.1  # the weighting is in effect
    for (gW, gb), (oW, ob) in zip(g, go):
        assert np.max(np.abs(gW - oW)) <= 1e-4 * np.max(np.abs(oW)) + 1e-12
        assert np.max(np.abs(gb - ob)) <= 1e-4 * np.max(np.abs(ob)) + 1e-12


def test_adam_step_matches_oracle(chem):
    net = capi.Mlp(chem, 10, 5, hidden=32, layers=2, seed=1)
    X, T, w = data(256, 10, 5, net.in_pad, net.out_pad, seed=2)
    p = [(W.astype(np.float64).copy(), b.astype(np.float64).copy()) for W, b in net.get()]
    ms = [(np.zeros_like(W), np.zeros_like(b)) for W, b in p]
    vs = [(np.zeros_like(W), np.zeros_like(b)) for W, b in p]
    for step in (1, 2, 3):
        _, g = net.grad(X, T, w)
        net.adam_step(1e-2)
        for (W, b), (gW, gb), (mW, mb), (vW, vb) in zip(p, g, ms, vs):
            mo.adam_step(W, gW.astype(np.float64), mW, vW, step, 1e-2)
            mo.adam_step(b, gb.astype(np.float64), mb, vb, step, 1e-2)
    for (W, b), (Wg, bg) in zip(p, net.get()):
        assert np.max(np.abs(W - Wg)) < 1e-5
        assert np.max(np.abs(b - bg)) < 1e-5


def test_training_fits_a_smooth_map(chem):
    rng = np.random.default_rng(7)
    net = capi.Mlp(chem, 8, 4, hidden=64, layers=3, seed=5)
    X = np.zeros((16384, net.in_pad), np.float32)
    X[:, :8] = rng.uniform(-1, 1, (16384, 8))
    T = np.zeros((16384, net.out_pad), np.float32)
    T[:, 0] = np.sin(X[:, 0] * 2) * X[:, 1]
    T[:, 1] = X[:, 2] ** 2 - X[:, 3]
    T[:, 2] = np.tanh(X[:, 4] + X[:, 5])
    T[:, 3] = X[:, 6] * X[:, 7]
    w = np.zeros(net.out_pad, np.float32)
    w[:4] = 1.0
    losses = net.train(X, T, w, epochs=30, batch=512, lr=3e-3)
    assert losses[-1] < 0.02 * losses[0]
