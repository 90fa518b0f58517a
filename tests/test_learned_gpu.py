"""The learned proposal network on the GPU against the FP64 oracle
(oracle/learned_oracle.py): tcgen05 forward, backward gradient, and training."""
import numpy as np
import pytest

import learned_oracle as LO
from scemc import learned

pytestmark = pytest.mark.gpu


def _rows(n, seed, field=None, kt_range=(0.2, 2.0)):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 14, 3))
    v /= np.linalg.norm(v, axis=2, keepdims=True)
    X = np.zeros((n, 43), np.float32)
    X[:, :42] = v.reshape(n, 42)
    X[:, 42] = rng.uniform(*kt_range, n)
    Y = rng.standard_normal((n, 3))
    Y /= np.linalg.norm(Y, axis=1, keepdims=True)
    return X, Y.astype(np.float32)


def _pad(X):
    Xp = np.zeros((X.shape[0], 64))
    Xp[:, :43] = X
    return Xp


def _perturbed(net, seed):
    rng = np.random.default_rng(seed)
    P = learned.unpack(net.params().copy())
    for k in P:
        P[k] += 0.2 * rng.standard_normal(P[k].shape).astype(np.float32) * (np.abs(P[k]).max() + 0.05)
    P["W1"][:, 43:] = 0
    P["W3"][20:] = 0
    P["b3"][20:] = 0
    flat = learned.pack(P)
    net.set_params(flat)
    return {k: v.astype(np.float64) for k, v in learned.unpack(flat).items()}


def test_forward_matches_oracle(gpu):
    net = learned.ProposalNet(seed=1)
    P = _perturbed(net, 2)
    X, _ = _rows(300, 3)  # not a multiple of 128: the tail tile is padded
    out = net.forward(X)
    ref = LO.forward(P, _pad(X), bf16=True)["o"][:, :20]
    err = np.abs(out - ref).max() / np.abs(ref).max()
    assert err < 2e-3, err


def test_gradient_matches_oracle(gpu):
    net = learned.ProposalNet(seed=4)
    P = _perturbed(net, 5)
    X, Y = _rows(256, 6)
    loss, g = net.loss_grad(X, Y)
    loss_ref, gref = LO.nll_and_grad(P, _pad(X), Y, bf16=True)
    assert loss == pytest.approx(loss_ref, rel=2e-3)
    G = learned.unpack(g)
    for k in gref:
        a, b = G[k].astype(np.float64).ravel(), gref[k].ravel()
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert rel < 3e-2 and cos > 0.999, (k, rel, cos)


def test_training_learns_a_local_field_conditional(gpu):
    """Targets drawn from the exact conditional of a Heisenberg site, a vMF with
    mean along the summed neighbour spins and kappa = J |h| / kT: training must
    bring the loss close to that conditional's entropy."""
    rng = np.random.default_rng(7)
    n = 8192
    X, _ = _rows(n, 8, kt_range=(0.5, 2.0))
    h = X[:, :42].reshape(n, 14, 3)[:, :8].sum(axis=1) * 0.25  # J = 0.25 meV on the 8 NN
    kap = np.linalg.norm(h, axis=1) / X[:, 42]
    mu = h / np.linalg.norm(h, axis=1, keepdims=True)
    Y = np.zeros((n, 3), np.float32)
    for i in range(n):
        o = np.zeros(32)
        o[0] = 50.0
        o[1:4] = mu[i]
        # softplus^-1(kappa * kT - 1e-3 kT) so that the head reproduces kappa exactly
        target = max((kap[i] - LO.KAPPA_MIN) * X[i, 42], 1e-6)
        o[4] = np.log(np.expm1(target)) if target < 20 else target
        Y[i], _ = LO.sample(o, X[i, 42], rng.random(), rng.random(), rng.random())
    # entropy of the true conditional: mean of -log f(y)
    H = -np.mean(LO.log_vmf(Y.astype(np.float64), mu[:, None, :], kap[:, None] + 0 * LO.KAPPA_MIN)[:, 0])
    net = learned.ProposalNet(seed=9)
    l0, _ = net.loss_grad(X[:1024], Y[:1024])
    losses = net.train(X, Y, batch=1024, epochs=100, lr=2e-3, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < l0 - 0.3
    assert losses[-1] < H + 0.25, (losses[-1], H)
