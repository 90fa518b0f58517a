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


def fcc_small(n):
    """The fcc l <= 2 + triangles + Zeeman model with the 18-site (12 + 6) environment."""
    w = models.config5_fcc(n=n)
    H = scemc.TiledHamiltonian(4, w.terms, dims=(n, n, n), magmoms=w.magmoms, field=w.field)
    OH = O.OracleHamiltonian(4, w.terms, (n, n, n), magmoms=w.magmoms, field=w.field)
    env = learned.environment_table(models.FCC.positions, (n, n, n))
    return w, H, OH, env


def env_rows(env, colors, pre, post, s_list, kt_mev):
    """Network inputs as the device saw them: an environment site of an earlier
    colour already carries this pass's decision."""
    k = env.shape[1]
    X = np.zeros((len(s_list), 3 * k + 1), np.float32)
    for i, s in enumerate(s_list):
        v = [post[t] if colors[t] < colors[s] else pre[t] for t in env[s]]
        X[i, :3 * k] = np.asarray(v, np.float32).reshape(-1)
        X[i, 3 * k] = kt_mev
    return X


@pytest.mark.parametrize("lattice,kernel", [("bcc", 2), ("bcc", 3), ("fcc", 2), ("fcc", 3)])
def test_learned_pass_replay(gpu, lattice, kernel):
    """bcc body-4 with the 14-site environment (43 inputs) and fcc l <= 2 with the
    18-site environment (55 inputs)."""
    w, H, OH, env = c4_small(4) if lattice == "bcc" else fcc_small(3)
    gH = scemc.GPUTiledHamiltonian(H)
    net = learned.ProposalNet(seed=3, n_env=env.shape[1])
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
        n0 = b.launches()
        b.run(1, kernel=kernel, proposals=3, mode=1)
        # kernel 3 decides inside the fused network kernel: one launch per colour
        assert b.launches() - n0 == H.n_colors * (1 if kernel == 3 else 2) + 1
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
            assert np.max(np.abs(prop[s] - x.astype(np.float32))) <= 3e-5, (s, prop[s], x)
            assert u[s] == O.philox_uniform(b1[2], b1[3])
        lq_ref = LO.log_q(out, tau, pre) - LO.log_q(out, tau, prop.astype(np.float64))
        np.testing.assert_allclose(lqr, lq_ref, rtol=0, atol=2e-4)  # FP32 mixture on the device
        # Metropolis-Hastings decisions, near-threshold ties flagged
        la = -beta * dE64 + lqr
        oacc = (la >= 0) | (u < np.exp(np.minimum(la, 0.0)))
        tie = (np.abs(la - np.log(u)) <= beta * tol) | (np.abs(la) <= beta * tol)
        mism = (flag == 1) != oacc
        assert not (mism & ~tie).any(), np.nonzero(mism & ~tie)[0][:5]
        ties += int((mism & tie).sum())
        att += H.n_sites
    assert ties <= max(1, att // 100)


def test_learned_fcc_pass_and_or_replay_at_many_wave_size(gpu):
    """The learned + overrelaxation form of the large frustrated configuration at a
    size whose colours fill many waves (fcc 48^3 x 4 sites, 32 rungs, kT geometric in
    [0.05, 2.0] meV, 18-site environment): one learned Metropolis-Hastings pass (the
    fused network + decision kernel) and one overrelaxation pass through the forms the
    library picks (two replicas per thread, one thread per item, no prefetch), recorded
    on rung 17 (the second lane of thread 1) and replayed through the oracles: dE and
    the decisions at every site, the draws and the density ratio at 2000 sampled sites,
    the overrelaxation reflection at every site."""
    n = 48
    w = models.config5_fcc(n=n, replicas=32)
    H = w.hamiltonians()[0]
    OH = O.OracleHamiltonian(4, w.terms, (n, n, n), magmoms=w.magmoms, field=w.field)
    env = learned.environment_table(models.FCC.positions, (n, n, n))
    gH = scemc.GPUTiledHamiltonian(H)
    net = learned.ProposalNet(seed=3, n_env=env.shape[1])
    R, rec = 32, 17
    seeds = [0xF00D + 5 * r for r in range(R)]
    base = models.random_config(H.n_sites, 5)
    b = scemc.GPUBatch([gH], [R], [np.roll(base, 11 * r, axis=0) for r in range(R)], seeds, 0.6)
    b.set_betas(1.0 / w.kts)
    b.set_learned(net, env)
    b.record_slot(0, rec)
    beta = 1.0 / w.kts[rec]
    kt_mev = np.float32(1e3 / beta)
    colors = np.asarray(H.colors)
    pre = b.download()["configs"][rec].copy()
    cfg = pre.copy()
    b.record(True)
    b.run(1, kernel=3, proposals=3, mode=1, or_per_metropolis=1)
    # learned Metropolis-Hastings pass
    prop, u, dE32, flag = b.fetch_record(-1)
    lqr = b.fetch_record_ratio()
    assert np.all(flag != 3)
    dE64, scale, _, _ = OH.replay_sweep(cfg, prop.astype(np.float64), u, (flag == 1).astype(np.uint8), beta)
    mid = cfg.copy()
    tol = 1e-5 * scale + 1e-30
    assert np.all(np.abs(dE32.astype(np.float64) - dE64) <= tol)
    la = -beta * dE64 + lqr
    oacc = (la >= 0) | (u < np.exp(np.minimum(la, 0.0)))
    tie = (np.abs(la - np.log(u)) <= beta * tol) | (np.abs(la) <= beta * tol)
    mism = (flag == 1) != oacc
    assert not (mism & ~tie).any(), np.nonzero(mism & ~tie)[0][:5]
    ties = int((mism & tie).sum())
    sites = np.sort(np.random.default_rng(7).choice(H.n_sites, 2000, replace=False))
    X = env_rows(env, colors, pre, mid, sites, kt_mev)
    out = np.zeros((len(sites), 32))
    out[:, :20] = net.forward(X)
    for i, s in enumerate(sites):
        b0 = O.philox_block(seeds[rec], int(s) + 1, 1, 0, tag=4)
        b1 = O.philox_block(seeds[rec], int(s) + 1, 1, 1, tag=4)
        x, _ = LO.sample(out[i], float(kt_mev), O.philox_uniform(b0[0], b0[1]), O.philox_uniform(b0[2], b0[3]),
                         O.philox_uniform(b1[0], b1[1]))
        assert np.max(np.abs(prop[s] - x.astype(np.float32))) <= 3e-5, (s, prop[s], x)
        assert u[s] == O.philox_uniform(b1[2], b1[3])
    tau = np.full(len(sites), float(kt_mev))
    lq_ref = LO.log_q(out, tau, pre[sites]) - LO.log_q(out, tau, prop[sites].astype(np.float64))
    np.testing.assert_allclose(lqr[sites], lq_ref, rtol=0, atol=2e-4)
    # overrelaxation pass on the state the learned pass left
    prop, u, dE32, flag = b.fetch_record(0)
    pre_or = cfg.copy()
    dE64, scale, oacc, c = OH.replay_sweep(cfg, prop.astype(np.float64), u, (flag == 1).astype(np.uint8), beta,
                                           want_c=True)
    att = (flag == 0) | (flag == 1)
    tol = 1e-5 * scale + 1e-30
    assert np.all(np.abs(dE32[att].astype(np.float64) - dE64[att]) <= tol[att])
    with np.errstate(divide="ignore"):
        thr = -np.log(u) / beta
    tie = (np.abs(dE64 - thr) <= tol) | (np.abs(dE64) <= tol)
    mism = att & ((flag == 1) != oacc)
    assert not (mism & ~tie).any(), np.nonzero(mism & ~tie)[0][:5]
    ties += int((mism & tie).sum())
    h = c[:, [3, 1, 2]]
    a = h / np.linalg.norm(h, axis=1, keepdims=True)
    refl = 2.0 * np.sum(pre_or * a, axis=1, keepdims=True) * a - pre_or
    refl /= np.linalg.norm(refl, axis=1, keepdims=True)
    assert np.max(np.abs(prop[att] - refl[att])) <= 1e-4
    np.testing.assert_array_equal(b.download()["configs"][rec], cfg)
    E_or = OH.total_energy(cfg)
    assert abs(b.total_energy(rec) - E_or) <= 1e-10 * max(1.0, abs(E_or))
    assert ties <= max(1, 2 * H.n_sites // 100)


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
    """The learned proposal trained on plain-chain environments (bcc 8^3 with the
    J1/J2 + body-4 model, 8 chains at kT = 0.3 meV, ordered phase, every chain started
    from the ordered state): higher acceptance and a shorter integrated
    autocorrelation time of E than adaptive-step Metropolis; the same energy from
    the row-parallel and replica-parallel kernels and, within the spread of the
    chains, from plain Metropolis. (Exactness of the Hastings step itself is pinned
    by the dimer and field tests; a plain chain's long-wavelength modes relax slowly,
    so the plain comparison uses the chain-to-chain spread and a longer warm-up.)"""
    n = 8
    w = models.config4_bcc_body4(n)
    H = scemc.TiledHamiltonian(2, w.terms, dims=(n, n, n))
    gH = scemc.GPUTiledHamiltonian(H)
    env = learned.environment_table(models.BCC.positions, (n, n, n))
    kts = np.full(8, 0.3 * MEV)
    up = np.tile([0.0, 0.0, 1.0], (H.n_sites, 1))
    X, Y = learned.collect_training_set(gH, env, kts, 65536, sweeps_therm=500, snapshots=16, spacing=20, seed=1,
                                        init=up)
    net = learned.ProposalNet(seed=5)
    losses = net.train(X, Y, batch=1024, epochs=40, lr=2e-3, seed=2)
    assert np.all(np.isfinite(losses)) and losses[-1] < losses[0], losses[[0, -1]]
    kw = dict(kT=kts, exchange=False, sweeps_measure=10000, seed=11, init=up)
    plain = scemc.gpu_run_pt(gH, sweeps_therm=4000, **kw)
    runs = {k: scemc.gpu_run_pt(gH, learned=(net, env), proposals=3, kernel=k, sweeps_therm=1000, **kw)
            for k in (2, 3)}

    def summary(r):
        e = np.array([p.stats["energy"].mean[0] for p in r.points])
        return e.mean(), e.std(ddof=1) / math.sqrt(len(e)), np.mean([p.acceptance_metropolis for p in r.points]), \
            np.mean([p.stats["energy"].tau_int[0] for p in r.points])

    ep, sp, ap, tp = summary(plain)
    e2, s2, a2, t2 = summary(runs[2])
    e3, s3, a3, t3 = summary(runs[3])
    assert abs(e2 - e3) < 4 * math.hypot(s2, s3), (e2, e3, s2, s3)
    assert abs(e3 - ep) < 5 * math.hypot(s3, sp), (e3, ep, s3, sp)
    assert abs(a2 - a3) < 0.01 and a3 > ap, (a2, a3, ap)
    assert t3 < 0.5 * tp, (t3, tp)


@pytest.mark.parametrize("kernel", [2, 3])
def test_learned_dimer_is_exact_with_a_sharp_network(gpu, kernel):
    """An interacting case with a closed form: the dimer E = J e1.e2 has
    <E> = J L(beta |J|) (test_gpu_pt.jl:13-42). Each spin's proposal is a sharp
    (kappa ~ 8) mixture about directions that the network computes from the other
    spin, so the Hastings ratio carries the whole correction."""
    J = -0.02
    H = models.dimer(J=J)
    gH = scemc.GPUTiledHamiltonian(H)
    env = np.zeros((4, 14), np.int32)
    env[0, :] = 1  # site 1's environment is site 2 (and vice versa); sites 3, 4 are inactive
    net = learned.ProposalNet(seed=8)
    P = learned.unpack(net.params().copy())
    P["b3"][4:20:5] = 50.0  # softplus ~ 50: kappa = 50 / kT[meV] ~ 8 at kT = 6 meV
    net.set_params(learned.pack(P))
    kt = abs(J) / 3.0
    R = 32
    b = scemc.GPUBatch([gH], [R], [models.random_config(4, 70 + r) for r in range(R)], list(range(500, 500 + R)),
                       0.6)
    b.set_betas(np.full(R, 1.0 / kt))
    b.set_learned(net, env)
    b.run(500, proposals=3, kernel=kernel)
    es = []
    for _ in range(2000):
        b.run(5, proposals=3, kernel=kernel)
        es.append(b.download()["energies"].copy())
    es = np.asarray(es)
    m = es.mean()
    err = es.mean(axis=0).std(ddof=1) / math.sqrt(R)
    exact = J * langevin(abs(J) / kt)
    assert abs(m - exact) < 4 * err + 1e-4 * abs(J), (m, exact, err)
    cnt = b.download()["counters"]
    acc = cnt[:, 0].sum() / cnt[:, 1].sum()
    assert 0.01 < acc < 0.9, acc


def test_site_coeffs_match_the_oracle(gpu):
    """scemc_batch_site_coeffs (the field-mode network inputs) against the oracle's
    leave-one-out coefficients of the same spins, to the FP32 walk's accuracy."""
    for lattice in ("bcc", "fcc"):
        w, H, OH, _ = c4_small(4) if lattice == "bcc" else fcc_small(3)
        gH = scemc.GPUTiledHamiltonian(H)
        b = scemc.GPUBatch([gH], [2], [models.random_config(H.n_sites, 5), models.random_config(H.n_sites, 6)],
                           [1, 2], 0.6)
        for slot in (0, 1):
            c = b.site_coeffs(slot).astype(np.float64)
            cfg = b.download()["configs"][slot]
            z = OH.zrows(cfg)
            ref = np.array([OH.site_coeffs(s + 1, z)[1:] for s in range(H.n_sites)])
            scale = np.abs(ref).sum(axis=1, keepdims=True) + 1e-30
            assert np.max(np.abs(c - ref) / scale) < 1e-5, (lattice, slot)


def test_learned_field_pass_replay(gpu):
    """A field-mode learned pass (the network reads each item's coefficients in meV and
    kT) on the fcc l <= 2 model, kernel 3: dE and the Hastings decisions at every site
    (with the recorded density ratio), and the draws and the ratio recomputed from the
    network on the oracle's coefficients (their BF16 rounding can differ from the
    device's FP32 ones at a rounding boundary, so 99 % of the sites must match)."""
    w, H, OH, _ = fcc_small(3)
    gH = scemc.GPUTiledHamiltonian(H)
    net = learned.ProposalNet(seed=3, field_rows=8)
    seeds = [0xABC, 0xDEF]
    kts = np.array([0.5, 1.5]) * MEV
    b = scemc.GPUBatch([gH], [2], [models.random_config(H.n_sites, 1), models.random_config(H.n_sites, 2)], seeds,
                       0.6)
    b.set_betas(1.0 / kts)
    b.set_learned(net, None)
    beta = 1.0 / kts[0]
    kt_mev = np.float32(1e3 / beta)
    matched = total = 0
    for sw in range(1, 4):
        pre = b.download()["configs"][0].copy()
        cfg = pre.copy()
        b.record(True)
        b.run(1, kernel=3, proposals=3, mode=1)
        prop, u, dE32, flag = b.fetch_record(-1)
        lqr = b.fetch_record_ratio()
        assert np.all(flag != 3)
        dE64, scale, _, c = OH.replay_sweep(cfg, prop.astype(np.float64), u, (flag == 1).astype(np.uint8), beta,
                                            want_c=True)
        np.testing.assert_array_equal(b.download()["configs"][0], cfg)
        tol = 1e-5 * scale + 1e-30
        assert np.all(np.abs(dE32.astype(np.float64) - dE64) <= tol)
        la = -beta * dE64 + lqr
        oacc = (la >= 0) | (u < np.exp(np.minimum(la, 0.0)))
        tie = (np.abs(la - np.log(u)) <= beta * tol) | (np.abs(la) <= beta * tol)
        assert not (((flag == 1) != oacc) & ~tie).any()
        X = np.zeros((H.n_sites, 9), np.float32)
        X[:, :8] = 1.0e3 * c[:, 1:]
        X[:, 8] = kt_mev
        out = np.zeros((H.n_sites, 32))
        out[:, :20] = net.forward(X)
        tau = np.full(H.n_sites, float(kt_mev))
        lq_ref = LO.log_q(out, tau, pre) - LO.log_q(out, tau, prop.astype(np.float64))
        for s in range(H.n_sites):
            b0 = O.philox_block(seeds[0], s + 1, sw, 0, tag=4)
            b1 = O.philox_block(seeds[0], s + 1, sw, 1, tag=4)
            x, _ = LO.sample(out[s], float(kt_mev), O.philox_uniform(b0[0], b0[1]), O.philox_uniform(b0[2], b0[3]),
                             O.philox_uniform(b1[0], b1[1]))
            total += 1
            if np.max(np.abs(prop[s] - x.astype(np.float32))) <= 3e-5 and abs(lqr[s] - lq_ref[s]) <= 2e-4:
                matched += 1
            assert u[s] == O.philox_uniform(b1[2], b1[3])
    assert matched >= 0.99 * total, (matched, total)


def test_learned_field_moments_in_a_field_are_exact(gpu):
    """Field mode, moments in a field (vanishing bonds set the colouring): whatever the
    untrained network proposes from the coefficients, Metropolis-Hastings samples
    exp(-beta E): <E> per site = -h L(beta h)."""
    n = 4
    terms = models.heisenberg_pairs(models.BCC, [1e-12 * MEV, 1e-12 * MEV])
    H = scemc.TiledHamiltonian(2, terms, dims=(n, n, n), magmoms=[2.0, 2.0], field=[0.0, 0.0, 1.0])
    gH = scemc.GPUTiledHamiltonian(H)
    up = np.tile([0.0, 0.0, 1.0], (H.n_sites, 1))
    OH = O.OracleHamiltonian(2, terms, (n, n, n), magmoms=[2.0, 2.0], field=[0.0, 0.0, 1.0])
    h = (OH.total_energy(-up) - OH.total_energy(up)) / (2 * H.n_sites)
    net = learned.ProposalNet(seed=22, field_rows=3)
    P = learned.unpack(net.params().copy())
    P["W3"] *= 0.1
    P["b3"][4:20:5] = -3.0
    net.set_params(learned.pack(P))
    R = 8
    bh = 2.0
    b = scemc.GPUBatch([gH], [R], [models.random_config(H.n_sites, 10 + r) for r in range(R)],
                       list(range(200, 200 + R)), 0.6)
    b.set_betas(np.full(R, bh / h))
    b.set_learned(net, None)
    b.run(200, proposals=3, kernel=3)
    es = []
    for _ in range(300):
        b.run(5, proposals=3, kernel=3)
        es.append(b.download()["energies"].copy())
    es = np.asarray(es) / H.n_sites
    m = es.mean()
    err = es.mean(axis=0).std(ddof=1) / math.sqrt(R)
    assert abs(m - (-h * langevin(bh))) < max(4 * err, 2e-3 * h), (m, -h * langevin(bh), err)


def test_learned_field_dimer_is_exact(gpu):
    """Field mode on the interacting dimer E = J e1.e2, <E> = J L(beta |J|)
    (test_gpu_pt.jl:13-42): each spin's proposal is a sharp mixture about directions
    the network computes from its coefficients (J times the other spin) and kT, so the
    Hastings ratio carries the whole correction."""
    J = -0.02
    H = models.dimer(J=J)
    gH = scemc.GPUTiledHamiltonian(H)
    net = learned.ProposalNet(seed=8, field_rows=3)
    P = learned.unpack(net.params().copy())
    P["b3"][4:20:5] = 50.0  # softplus ~ 50: kappa = 50 / kT[meV] ~ 8 at kT = 6.7 meV
    net.set_params(learned.pack(P))
    kt = abs(J) / 3.0
    R = 32
    b = scemc.GPUBatch([gH], [R], [models.random_config(4, 90 + r) for r in range(R)], list(range(700, 700 + R)),
                       0.6)
    b.set_betas(np.full(R, 1.0 / kt))
    b.set_learned(net, None)
    b.run(500, proposals=3, kernel=3)
    es = []
    for _ in range(2000):
        b.run(5, proposals=3, kernel=3)
        es.append(b.download()["energies"].copy())
    es = np.asarray(es)
    m = es.mean()
    err = es.mean(axis=0).std(ddof=1) / math.sqrt(R)
    exact = J * langevin(abs(J) / kt)
    assert abs(m - exact) < 4 * err + 1e-4 * abs(J), (m, exact, err)
    cnt = b.download()["counters"]
    acc = cnt[:, 0].sum() / cnt[:, 1].sum()
    assert 0.01 < acc < 0.95, acc
    for r in range(R):  # the running energy (FP32 dE over ~10^4 moves) tracks the FP64 recompute
        assert abs(b.download()["energies"][r] - b.total_energy(r)) <= 1e-5 * abs(J)
