"""Oracle (test infrastructure only) for the learned von Mises-Fisher mixture proposal.

FP64 numpy restatement of what the CUDA path computes: the per-site MLP
(43 -> 128 -> 128 -> 20, SiLU, inputs padded to 64 and outputs to 32), the
4-component vMF mixture head, its negative log-likelihood and the analytic
gradient of that loss with respect to every weight and bias, the mixture
sampler, and the Metropolis-Hastings acceptance with the proposal-density ratio.

The reference has no learned proposal (it is new in this build); the acceptance
rule follows the reference's Metropolis test in src/updates.jl:37-64 with the
Hastings factor q(e | env) / q(e' | env) added, so the stationary distribution is
the same Boltzmann distribution. The gradient is pinned here by central finite
differences (tests/test_learned_oracle.py); the GPU kernels are checked against
this file, never the other way round, and nothing in the product imports it.
"""
from __future__ import annotations

import math

import numpy as np

N_IN, N_IN_PAD, N_HID, N_OUT, N_OUT_PAD, N_COMP = 43, 64, 128, 20, 32, 4
KAPPA_MIN = 1e-3


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def softplus(x):
    return np.where(x > 20.0, x, np.log1p(np.exp(np.minimum(x, 20.0))))


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def init_params(seed: int, n_in: int = N_IN):
    """He-style initial weights (FP32 master copies, padded shapes): W1 (128, 64)
    with input columns n_in..63 zero, W2 (128, 128), W3 (32, 128) with output rows
    20..31 zero, biases zero. The concentration outputs start near softplus(1)."""
    rng = np.random.default_rng(seed)
    W1 = np.zeros((N_HID, N_IN_PAD))
    W1[:, :n_in] = rng.standard_normal((N_HID, n_in)) * math.sqrt(2.0 / n_in)
    W2 = rng.standard_normal((N_HID, N_HID)) * math.sqrt(2.0 / N_HID)
    W3 = np.zeros((N_OUT_PAD, N_HID))
    W3[:N_OUT] = rng.standard_normal((N_OUT, N_HID)) * math.sqrt(1.0 / N_HID) * 0.1
    b1, b2, b3 = np.zeros(N_HID), np.zeros(N_HID), np.zeros(N_OUT_PAD)
    b3[4:N_OUT:5] = 1.0
    return {k: v.astype(np.float32) for k, v in dict(W1=W1, b1=b1, W2=W2, b2=b2, W3=W3, b3=b3).items()}


def bf16_round(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    a = (a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000
    return a.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(P, X, bf16: bool = False):
    """X (n, 64) -> dict of pre-activations, activations and outputs (FP64). With
    bf16=True the inputs, weights and hidden activations are rounded to BF16 where
    the tensor-core path stores them (products and sums stay exact)."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    X = r(X)
    z1 = X @ r(P["W1"]).T + P["b1"]
    h1 = r(silu(z1))
    z2 = h1 @ r(P["W2"]).T + P["b2"]
    h2 = r(silu(z2))
    o = h2 @ r(P["W3"]).T + P["b3"]
    return dict(X=X, z1=z1, h1=h1, z2=z2, h2=h2, o=o)


def head(o, tau):
    """Mixture parameters from the 20 outputs: weights pi (softmax of the logits),
    unit means mu, concentrations kappa = softplus(c) / tau + KAPPA_MIN where tau is
    kT in meV (the 43rd input), so the net predicts kappa * kT."""
    o = np.asarray(o, np.float64)
    a = o[:, 0:N_OUT:5]
    m = np.stack([o[:, 5 * k + 1:5 * k + 4] for k in range(N_COMP)], axis=1)  # (n, 4, 3)
    c = o[:, 4:N_OUT:5]
    amax = a.max(axis=1, keepdims=True)
    lse = amax[:, 0] + np.log(np.exp(a - amax).sum(axis=1))
    logpi = a - lse[:, None]
    mn = np.linalg.norm(m, axis=2)
    mu = m / np.maximum(mn, 1e-12)[:, :, None]
    kappa = softplus(c) / np.asarray(tau, np.float64)[:, None] + KAPPA_MIN
    return logpi, mu, mn, kappa, c


def log_vmf(x, mu, kappa):
    """log density on S^2: log kappa - log 2pi - log(1 - e^{-2 kappa}) + kappa (mu.x - 1)."""
    d = np.einsum("nkc,nc->nk", mu, x)
    return np.log(kappa) - math.log(2 * math.pi) - np.log(-np.expm1(-2.0 * kappa)) + kappa * (d - 1.0)


def log_q(o, tau, x):
    logpi, mu, _, kappa, _ = head(o, tau)
    l = logpi + log_vmf(np.asarray(x, np.float64), mu, kappa)
    lm = l.max(axis=1, keepdims=True)
    return lm[:, 0] + np.log(np.exp(l - lm).sum(axis=1))


def nll_and_grad(P, X, Y, bf16: bool = False, n_in: int = N_IN):
    """Mean negative log-likelihood of the unit targets Y (n, 3) and its gradient
    for every parameter (same shapes as P); bf16 as in forward(). Column n_in - 1
    of X is kT."""
    f = forward(P, X, bf16)
    n = X.shape[0]
    tau = np.asarray(X, np.float64)[:, n_in - 1]  # the head reads kT unrounded
    o = f["o"]
    logpi, mu, mn, kappa, c = head(o, tau)
    Y = np.asarray(Y, np.float64)
    lf = log_vmf(Y, mu, kappa)
    l = logpi + lf
    lm = l.max(axis=1, keepdims=True)
    lq = lm[:, 0] + np.log(np.exp(l - lm).sum(axis=1))
    r = np.exp(l - lq[:, None])  # responsibilities
    pi = np.exp(logpi)
    do = np.zeros_like(o)
    d = np.einsum("nkc,nc->nk", mu, Y)
    # d(-log q)/d logits
    do[:, 0:N_OUT:5] = pi - r
    # d/d kappa of log f: 1/kappa - 2/(e^{2 kappa} - 1) + (mu.y - 1)
    dlf_dk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (d - 1.0)
    do[:, 4:N_OUT:5] = -r * dlf_dk * sigmoid(c) / tau[:, None]
    for k in range(N_COMP):
        g = kappa[:, k, None] * (Y - d[:, k, None] * mu[:, k])  # (I - mu mu^T) kappa y
        do[:, 5 * k + 1:5 * k + 4] = -r[:, k, None] * g / np.maximum(mn[:, k, None], 1e-12)
    do /= n
    dW3 = do.T @ f["h2"]
    db3 = do.sum(axis=0)
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    dz2 = (do @ r(P["W3"])) * dsilu(f["z2"])
    dW2 = dz2.T @ f["h1"]
    db2 = dz2.sum(axis=0)
    dz1 = (dz2 @ r(P["W2"])) * dsilu(f["z1"])
    dW1 = dz1.T @ f["X"]
    db1 = dz1.sum(axis=0)
    grads = dict(W1=dW1, b1=db1, W2=dW2, b2=db2, W3=dW3, b3=db3)
    grads["W1"][:, n_in:] = 0.0
    grads["W3"][N_OUT:] = 0.0
    grads["b3"][N_OUT:] = 0.0
    return float(-lq.mean()), grads


def orthonormal_pair(mu):
    """(t1, t2) orthonormal and perpendicular to the unit vector mu: t1 from the
    coordinate axis least aligned with mu (Gram-Schmidt), t2 = mu x t1."""
    ax = np.argmin(np.abs(mu))
    e = np.zeros(3)
    e[ax] = 1.0
    t1 = e - mu[ax] * mu
    t1 /= np.linalg.norm(t1)
    t2 = np.cross(mu, t1)
    return t1, t2


def sample(o_row, tau, u_comp, u_w, u_phi):
    """One draw from the mixture of one site: component by inverse CDF of the
    weights, w = mu.x by the inverse CDF 1 + log(u + (1 - u) e^{-2 kappa}) / kappa,
    azimuth 2 pi u_phi about mu."""
    logpi, mu, _, kappa, _ = head(np.asarray(o_row)[None, :], np.array([tau]))
    pi = np.exp(logpi[0])
    k = 0
    acc = pi[0]
    while k < N_COMP - 1 and u_comp >= acc:
        k += 1
        acc += pi[k]
    kap = kappa[0, k]
    w = 1.0 + math.log(u_w + (1.0 - u_w) * math.exp(-2.0 * kap)) / kap
    w = min(1.0, max(-1.0, w))
    v = math.sqrt(max(0.0, 1.0 - w * w))
    t1, t2 = orthonormal_pair(mu[0, k])
    phi = 2.0 * math.pi * u_phi
    x = w * mu[0, k] + v * (math.cos(phi) * t1 + math.sin(phi) * t2)
    return x / np.linalg.norm(x), k


def mh_accept(beta, dE, logq_old, logq_new, u):
    """Metropolis-Hastings with the proposal ratio: accept when
    u < exp(-beta dE + log q(e_old) - log q(e_new)) (always when that is >= 0)."""
    la = -beta * dE + (logq_old - logq_new)
    return la >= 0.0 or u < math.exp(la)
