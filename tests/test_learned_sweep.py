"""The learned proposal inside the sweep (B200, -m gpu), against the oracle:
replay of a recorded learned Metropolis pass (the mixture draw from the keyed
stream, dE, the density ratio recomputed from the network and the Hastings
decision), and exactness of the stationary distribution for moments in a field
under an untrained network."""
import math

import numpy as np
import pytest

import learned_oracle as LO
import oracle as O
import scemc
from scemc import learned, models

pytestmark = pytest.mark.gpu

MEV = 1e-3


def c4_small(n):
    w = models.config4_bcc_body4(n)
    H = scemc.TiledHamiltonian(2, w.terms, dims=(n, n, n))
    OH = O.OracleHamiltonian(2, w.terms, (n, n, n))
    env = learned.environment_table(models.BCC.positions, (n, n, n))
    return w, H, OH, env


def env_rows(env, colors, pre, post, s_list, kt_mev):
    """Network inputs as the device saw them: an environment site of an earlier
    colour already carries this pass's decision."""
    X = np.zeros((len(s_list), 43), np.float32)
    for i, s in enumerate(s_list):
        v = [post[t] if colors[t] < colors[s] else pre[t] for t in env[s]]
        X[i, :42] = np.asarray(v, np.float32).reshape(-1)
        X[i, 42] = kt_mev
    return X


@pytest.mark.parametrize("kernel", [2, 3])
def test_learned_pass_replay(gpu, kernel):
    w, H, OH, env = c4_small(4)
    gH = scemc.GPUTiledHamiltonian(H)
    net = learned.ProposalNet(seed=3)
    seeds = [0xABC, 0xDEF]
    kts = np.array([0.5, 1.5]) * MEV
    b = scemc.GPUBatch([gH], [2], [models.random_config(H.n_sites, 1), models.random_config(H.n_sites, 2)], seeds,
                       0.6)
    b.set_betas(1.0 / kts)
    b.set_learned(net, env)
    beta = 1.0 / kts[0]
    kt_mev = np.float32(1e3 / beta)
    colors = np.asarray(H.colors)
    ties = att = 0
    for sw in range(1, 4):
        pre = b.download()["configs"][0].copy()
        cfg = pre.copy()
        b.record(True)
        b.run(1, kernel=kernel, proposals=3, mode=1)
        prop, u, dE32, flag = b.fetch_record(-1)
        lqr = b.fetch_record_ratio()
        assert np.all(flag != 3)
        dE64, scale, _, _ = OH.replay_sweep(cfg, prop.astype(np.float64), u, (flag == 1).astype(np.uint8), beta)
        post = b.download()["configs"][0]
        np.testing.assert_array_equal(post, cfg)
        tol = 1e-5 * scale + 1e-30
        assert np.all(np.abs(dE32.astype(np.float64) - dE64) <= tol)
        # the draws and the density ratio, recomputed from the same network
        sites = np.arange(H.n_sites)
        X = env_rows(env, colors, pre, post, sites, kt_mev)
        out = np.zeros((H.n_sites, 32))
        out[:, :20] = net.forward(X)
        tau = np.full(H.n_sites, float(kt_mev))
        for s in sites:
            b0 = O.philox_block(seeds[0], int(s) + 1, sw, 0, tag=4)
            b1 = O.philox_block(seeds[0], int(s) + 1, sw, 1, tag=4)
            x, _ = LO.sample(out[s], float(kt_mev), O.philox_uniform(b0[0], b0[1]), O.philox_uniform(b0[2], b0[3]),
                             O.philox_uniform(b1[0], b1[1]))
            assert np.max(np.abs(prop[s] - x.astype(np.float32))) <= 2e-6, (s, prop[s], x)
            assert u[s] == O.philox_uniform(b1[2], b1[3])
        lq_ref = LO.log_q(out, tau, pre.astype(np.float32).astype(np.float64)) - LO.log_q(out, tau,
                                                                                       prop.astype(np.float64))
        np.testing.assert_allclose(lqr, lq_ref, rtol=0, atol=1e-9)
        # Metropolis-Hastings decisions, near-threshold ties flagged
        la = -beta * dE64 + lqr
        oacc = (la >= 0) | (u < np.exp(np.minimum(la, 0.0)))
        tie = (np.abs(la - np.log(u)) <= beta * tol) | (np.abs(la) <= beta * tol)
        mism = (flag == 1) != oacc
        assert not (mism & ~tie).any(), np.nonzero(mism & ~tie)[0][:5]
        ties += int((mism & tie).sum())
        att += H.n_sites
    assert ties <= max(1, att // 100)


def langevin(x):
    return 1.0 / math.tanh(x) - 1.0 / x


def test_learned_moments_in_a_field_are_exact(gpu):
    """Moments coupled by vanishing bonds (they only set the colouring) in a field:
    whatever the network proposes, Metropolis-Hastings with its density ratio
    samples exp(-beta E): <E> per site = -h L(beta h)."""
    n = 4
    terms = models.heisenberg_pairs(models.BCC, [1e-12 * MEV, 1e-12 * MEV])
    H = scemc.TiledHamiltonian(2, terms, dims=(n, n, n), magmoms=[2.0, 2.0], field=[0.0, 0.0, 1.0])
    gH = scemc.GPUTiledHamiltonian(H)
    up = np.tile([0.0, 0.0, 1.0], (H.n_sites, 1))
    OH = O.OracleHamiltonian(2, terms, (n, n, n), magmoms=[2.0, 2.0], field=[0.0, 0.0, 1.0])
    h = (OH.total_energy(-up) - OH.total_energy(up)) / (2 * H.n_sites)
    assert h > 0
    env = learned.environment_table(models.BCC.positions, (n, n, n))
    net = learned.ProposalNet(seed=21)
    P = learned.unpack(net.params().copy())
    P["W3"] *= 0.1
    P["b3"][4:20:5] = -3.0  # broad components (kappa ~ 1) about network-chosen directions
    net.set_params(learned.pack(P))
    R = 8
    bh = 2.0
    b = scemc.GPUBatch([gH], [R], [models.random_config(H.n_sites, 10 + r) for r in range(R)],
                       list(range(100, 100 + R)), 0.6)
    b.set_betas(np.full(R, bh / h))
    b.set_learned(net, env)
    b.run(200, proposals=3, kernel=3)
    es = []
    for _ in range(300):
        b.run(5, proposals=3, kernel=3)
        es.append(b.download()["energies"].copy())
    es = np.asarray(es) / H.n_sites
    m = es.mean()
    err = es.mean(axis=0).std(ddof=1) / math.sqrt(R)
    assert abs(m - (-h * langevin(bh))) < max(4 * err, 2e-3 * h), (m, -h * langevin(bh), err)
    cnt = b.download()["counters"]
    assert cnt[:, 0].sum() > 0.05 * cnt[:, 1].sum()  # some learned proposals are accepted


def test_trained_network_beats_plain_metropolis(gpu):
    """The learned proposal trained on plain-chain environments (bcc 16^3 with the
    J1/J2 + body-4 model, ordered phase, both samplers started from the ordered
    state): higher acceptance and a shorter integrated autocorrelation time of E
    than adaptive-step Metropolis, the same energy within the error bars, and the
    same acceptance from the row-parallel and replica-parallel kernels."""
    n = 16
    w = models.config4_bcc_body4(n)
    H = scemc.TiledHamiltonian(2, w.terms, dims=(n, n, n))
    gH = scemc.GPUTiledHamiltonian(H)
    env = learned.environment_table(models.BCC.positions, (n, n, n))
    kts = np.array([0.3, 0.6]) * MEV
    up = np.tile([0.0, 0.0, 1.0], (H.n_sites, 1))
    X, Y = learned.collect_training_set(gH, env, kts, 131072, sweeps_therm=500, snapshots=16, spacing=20, seed=1,
                                        init=up)
    net = learned.ProposalNet(seed=5)
    losses = net.train(X, Y, batch=1024, epochs=40, lr=2e-3, seed=2)
    assert losses[-1] < losses[0] - 0.5, losses[[0, -1]]
    kw = dict(kT=kts, exchange=False, sweeps_therm=500, sweeps_measure=6000, seed=11, init=up)
    plain = scemc.gpu_run_pt(gH, **kw)
    runs = {k: scemc.gpu_run_pt(gH, learned=(net, env), proposals=3, kernel=k, **kw) for k in (2, 3)}
    for k, lrn in runs.items():
        for pp, pl in zip(plain.points, lrn.points):
            e0, s0 = pp.stats["energy"].mean[0], pp.stats["energy"].err[0]
            e1, s1 = pl.stats["energy"].mean[0], pl.stats["energy"].err[0]
            assert abs(e0 - e1) < 4 * math.hypot(s0, s1) + 1e-12, (k, e0, e1, s0, s1)
            assert pl.acceptance_metropolis > pp.acceptance_metropolis, (k, pl.acceptance_metropolis,
                                                                         pp.acceptance_metropolis, losses[-1])
    a2 = [p.acceptance_metropolis for p in runs[2].points]
    a3 = [p.acceptance_metropolis for p in runs[3].points]
    assert np.allclose(a2, a3, atol=0.02), (a2, a3)
    t_plain = plain.points[0].stats["energy"].tau_int[0]
    t_lrn = runs[3].points[0].stats["energy"].tau_int[0]
    assert t_lrn < 0.5 * t_plain, (t_lrn, t_plain)
