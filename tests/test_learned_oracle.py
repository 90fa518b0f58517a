"""The learned-proposal oracle pinned on its own mathematics (CPU only): the
analytic NLL gradient against central finite differences, the vMF density's
normalisation on S^2, the sampler's inverse CDF, and the Hastings acceptance."""
import math

import numpy as np
import pytest

import learned_oracle as LO


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, LO.N_IN_PAD))
    v = rng.standard_normal((n, 14, 3))
    v /= np.linalg.norm(v, axis=2, keepdims=True)
    X[:, :42] = v.reshape(n, 42)
    X[:, 42] = rng.uniform(0.2, 2.0, n)
    Y = rng.standard_normal((n, 3))
    Y /= np.linalg.norm(Y, axis=1, keepdims=True)
    return X, Y


def test_gradient_matches_finite_differences():
    P = {k: v.astype(np.float64) for k, v in LO.init_params(3).items()}
    rng = np.random.default_rng(1)
    for k in P:  # move off the symmetric start so every output channel matters
        P[k] = P[k] + 0.3 * rng.standard_normal(P[k].shape) * (np.abs(P[k]).max() + 0.1)
    P["W1"][:, LO.N_IN:] = 0.0
    P["W3"][LO.N_OUT:] = 0.0
    P["b3"][LO.N_OUT:] = 0.0
    X, Y = _batch(16, 2)
    _, g = LO.nll_and_grad(P, X, Y)
    h = 1e-6
    for name, idxs in [("W1", [(0, 0), (5, 42), (127, 13)]), ("b1", [(3,), (100,)]), ("W2", [(1, 2), (64, 127)]),
                       ("b2", [(7,)]), ("W3", [(0, 0), (4, 17), (13, 99), (19, 127)]), ("b3", [(0,), (4,), (9,), (18,)])]:
        for ix in idxs:
            Pp = {k: v.copy() for k, v in P.items()}
            Pm = {k: v.copy() for k, v in P.items()}
            Pp[name][ix] += h
            Pm[name][ix] -= h
            fd = (LO.nll_and_grad(Pp, X, Y)[0] - LO.nll_and_grad(Pm, X, Y)[0]) / (2 * h)
            assert g[name][ix] == pytest.approx(fd, rel=2e-5, abs=1e-8), (name, ix)


def test_vmf_density_normalised_and_sampler_inverse_cdf():
    rng = np.random.default_rng(0)
    # quadrature over S^2 of exp(log q) for a random mixture
    o = rng.standard_normal((1, LO.N_OUT_PAD)) * 2.0
    tau = np.array([0.7])
    nt, nph = 400, 800
    th = (np.arange(nt) + 0.5) * math.pi / nt
    ph = (np.arange(nph) + 0.5) * 2 * math.pi / nph
    T, PH = np.meshgrid(th, ph, indexing="ij")
    x = np.stack([np.sin(T) * np.cos(PH), np.sin(T) * np.sin(PH), np.cos(T)], axis=-1).reshape(-1, 3)
    lq = LO.log_q(np.repeat(o, x.shape[0], axis=0), np.repeat(tau, x.shape[0]), x)
    integral = (np.exp(lq) * np.sin(T).reshape(-1)).sum() * (math.pi / nt) * (2 * math.pi / nph)
    assert integral == pytest.approx(1.0, abs=2e-4)
    # samples: mean of mu.x for a single sharp component equals coth(k) - 1/k
    o1 = np.zeros(LO.N_OUT_PAD)
    o1[0] = 50.0  # component 0 takes all the weight
    o1[1:4] = [0.0, 0.0, 1.0]
    o1[4] = 3.0
    kap = float(LO.softplus(np.array([3.0]))[0] / 0.5 + LO.KAPPA_MIN)
    ws = []
    for i in range(4000):
        xs, k = LO.sample(o1, 0.5, rng.random(), rng.random(), rng.random())
        assert k == 0 and abs(np.linalg.norm(xs) - 1) < 1e-12
        ws.append(xs[2])
    assert np.mean(ws) == pytest.approx(1 / math.tanh(kap) - 1 / kap, abs=0.01)


def test_hastings_acceptance():
    assert LO.mh_accept(1.0, -1.0, 0.0, 0.0, 0.999)
    assert LO.mh_accept(1.0, 1.0, 2.0, 0.0, 0.999)  # ratio e^{1} >= 1
    assert not LO.mh_accept(1.0, 1.0, 0.0, 0.0, 0.5)  # e^{-1} = 0.37 < 0.5
    assert LO.mh_accept(1.0, 1.0, 0.0, 0.0, 0.3)
