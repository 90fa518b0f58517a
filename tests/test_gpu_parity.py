"""Parity of the CUDA sweep against the FP64 oracle (run on a B200: -m gpu).

Every gate calls libscemc_cuda.so through the C ABI (via the package's ctypes
API). Tolerances (the parity bar of this path):
  * per-proposal dE: |dE32 - dE64| <= 1e-5 * sum|c| (sum|znew| + sum|zold|)
    (the reference's scaled form, test_gpu.jl:168,174, with 1e-5 for FP32);
  * accept/reject: identical on replay, except near-threshold ties where the
    threshold -log(u)/beta (or 0) lies within that dE tolerance of dE64;
  * proposals: the FP32-rounded reference keyed proposal (<= 1 FP32 ulp);
  * total energy: FP64 device recompute within 1e-10 relative of the oracle;
  * statistics: within the combined log-binning / jackknife error bars.
"""
import math

import numpy as np
import pytest

import oracle as O
import scemc
from scemc import _lib, models

pytestmark = pytest.mark.gpu

ZB = (0.3, -1.2, 2.0)
F32_ULP = 2.0 ** -23

MODELS = {
    "dimer": (4, models.dimer_terms(), (1, 1, 1), {}),
    "dimer_zeeman": (4, models.dimer_terms(), (2, 1, 1), dict(magmoms=[2.2, 2.2, 1.0, 0.0], field=ZB)),
    "biquadratic": (2, models.biquadratic_terms(3), (2, 2, 2), {}),
    "biquadratic_zeeman": (2, models.biquadratic_terms(3), (2, 2, 2), dict(magmoms=[1.5, 0.7], field=ZB)),
    "zeeman_only": (2, [], (2, 2, 1), dict(magmoms=[1.0, 2.0], field=ZB)),
    "chain": (1, models.chain_terms(-0.05), (4, 4, 2), {}),
    "threebody": (1, models.threebody_terms(0.05), (4, 2, 2), {}),
    "fourbody": (1, models.fourbody_terms(0.03), (4, 2, 2), {}),
    "mixed": (2, models.mixed_terms(7), (2, 2, 1), {}),
    "high_l": (1, models.highl_terms(11, 4), (3, 2, 1), {}),
    "sc_J1J2": (1, models.config1_sc().terms, (4, 4, 4), {}),
    "bcc_l2_plaq_zeeman": (2, models.config2_bcc_l2().terms, (3, 3, 3), dict(magmoms=[2.0, 2.0], field=[0, 0, 1.0])),
    "bcc_triangles": (2, models.config3_bcc_pt().terms, (3, 3, 3), {}),
    "bcc_body4": (2, models.config4_bcc_body4().terms, (3, 3, 3), {}),
    "fcc_l2_tri_zeeman": (4, models.config5_fcc(n=2).terms, (2, 2, 2), dict(magmoms=[2.0] * 4, field=[0.3] * 3)),
    "bcc_l2_body3": (2, models.bcc_l2_body3(3).terms, (3, 3, 3), {}),
}


def build(name):
    nca, terms, dims, kw = MODELS[name]
    H = scemc.TiledHamiltonian(nca, terms, dims=dims, **kw)
    OH = O.OracleHamiltonian(nca, terms, dims, **kw)
    return H, OH


def rand_cfg(n, seed):
    return models.random_config(n, seed)


def energy_scale(H):
    """Typical |site energy| of a model: beta is chosen so moves are ~50/50."""
    return 0.05


def f32_normalised(v):
    v = np.asarray(v, np.float64)
    return (v / np.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])).astype(np.float32)


def check_pass(OH, cfg, rec, beta, kind, seed=None, sweep=None, step=None, orpass=0, sample=None):
    """Replays one recorded pass; returns (#ties, #attempted). cfg updated in place.
    dE and the decisions are checked at every site; the proposals at every site, or
    at `sample` random sites of a large lattice (the check is a Python loop)."""
    prop, u, dE32, flag = rec
    pre = cfg.copy()
    dev_acc = (flag == 1).astype(np.uint8)
    dE64, scale, oacc, c = OH.replay_sweep(cfg, prop.astype(np.float64), u, dev_acc, beta, want_c=True)
    active = OH.array("site_active").astype(bool)
    has_l1 = OH.array("site_has_l1").astype(bool)
    visited = flag != 3
    if kind == "metro":
        assert np.array_equal(visited, active)
    else:
        assert np.array_equal(visited, active & has_l1)
    att = visited & (flag != 2)
    tol = 1e-5 * scale + 1e-30
    # dE within the scaled FP32 tolerance
    bad = att & (np.abs(dE32.astype(np.float64) - dE64) > tol)
    assert not bad.any(), (np.nonzero(bad)[0][:5], dE32[bad][:5], dE64[bad][:5], scale[bad][:5])
    # accept/reject identical except flagged ties
    with np.errstate(divide="ignore"):
        thr = -np.log(u) / beta
    tie = (np.abs(dE64 - thr) <= tol) | (np.abs(dE64) <= tol)
    mism = att & ((flag == 1) != oacc)
    assert not (mism & ~tie).any(), np.nonzero(mism & ~tie)[0][:5]
    n_sites = len(flag)
    pick = np.arange(n_sites)
    if sample is not None and sample < n_sites:
        pick = np.sort(np.random.default_rng(sweep).choice(n_sites, sample, replace=False))
    if kind == "metro":
        for s in np.nonzero(active[pick])[0]:
            s = pick[s]
            b0 = O.philox_block(seed, int(s) + 1, sweep, 0)
            if O.philox_uniform(b0[0], b0[1]) < 0.2:
                exp = (-pre[s]).astype(np.float32)
            else:
                e2, _ = O.keyed_proposal(seed, int(s) + 1, sweep, pre[s], step)
                exp = f32_normalised(e2)
            assert np.max(np.abs(prop[s] - exp)) <= F32_ULP, (s, prop[s], exp)
    else:
        for s in np.nonzero(visited[pick])[0]:
            s = pick[s]
            h = np.array([c[s, 3], c[s, 1], c[s, 2]])
            hn = np.linalg.norm(h)
            if flag[s] == 2:
                assert hn < 1e-9
                continue
            a = h / hn
            e = pre[s]
            r = 2.0 * np.dot(e, a) * a - e
            exp = r / np.linalg.norm(r)
            assert np.max(np.abs(prop[s] - exp)) <= 1e-4, (s, prop[s], exp)
            b = O.philox_block(seed, int(s) + 1, sweep, orpass, tag=1)
            assert u[s] == O.philox_uniform(b[0], b[1])
    return int(tie[mism].sum()), int(att.sum()), n_sites


NOT_FAST = {"high_l"}  # programs outside the fast kinds (l >= 3 members)
FAST = [m for m in MODELS if m not in NOT_FAST]

# (model, lanes, mode, kernel, proposals): kernel 1 = generic record walk, 0 = auto
# (the row-parallel fast kernel wherever the model allows it), 3 = replica-parallel
# kernel; proposals 1 = precomputed before the colour loop, 2 = inline.
REPLAY_CASES = [(m, 4, 2, 1, 0) for m in MODELS] + [(m, 0, 2, 0, 1) for m in FAST] + [
    ("biquadratic", 1, 1, 1, 0), ("biquadratic", 32, 1, 1, 0), ("bcc_l2_plaq_zeeman", 1, 2, 1, 0),
    ("bcc_l2_plaq_zeeman", 32, 1, 1, 0), ("high_l", 1, 1, 0, 0), ("mixed", 32, 2, 0, 0),
    ("fourbody", 32, 2, 1, 0), ("sc_J1J2", 8, 1, 1, 0), ("fcc_l2_tri_zeeman", 16, 2, 1, 0),
    ("bcc_l2_plaq_zeeman", 0, 1, 0, 2), ("bcc_l2_plaq_zeeman", 0, 1, 0, 1), ("bcc_l2_plaq_zeeman", 0, 2, 0, 2),
    ("fcc_l2_tri_zeeman", 0, 1, 0, 2), ("threebody", 0, 1, 0, 1), ("chain", 0, 2, 0, 2),
    ("bcc_l2_plaq_zeeman", 0, 3, 0, 1), ("fcc_l2_tri_zeeman", 0, 3, 0, 2), ("biquadratic", 4, 3, 1, 0),
    ("mixed", 8, 3, 0, 0),
] + [(m, 0, 1, 3, 2) for m in FAST] + [("bcc_l2_plaq_zeeman", 0, 3, 3, 1), ("fcc_l2_tri_zeeman", 0, 3, 3, 2)] + [
    (m, 0, 4, 2, 2) for m in FAST] + [(m, 0, 1, 4, 2) for m in FAST] + [
    ("bcc_l2_plaq_zeeman", 0, 3, 4, 1), ("fcc_l2_tri_zeeman", 0, 1, 4, 1), ("bcc_body4", 0, 3, 4, 2)] + [
    (m, 0, 2, 3, 1 + (i % 2)) for i, m in enumerate(FAST)]


@pytest.mark.parametrize("name,lanes,mode,kernel,proposals", REPLAY_CASES,
                         ids=[f"{m}-G{g}-mode{d}-k{k}-p{q}" for m, g, d, k, q in REPLAY_CASES])
def test_sweep_replay(gpu, name, lanes, mode, kernel, proposals):
    H, OH = build(name)
    gH = scemc.GPUTiledHamiltonian(H)
    seed, step, beta = 0xC0FFEE + lanes, 0.6, 1 / 0.05
    n_or = 2 if H.site_has_l1.any() else 0
    b = scemc.GPUBatch([gH], [1], [rand_cfg(H.n_sites, 7)], [seed], step)
    b.set_betas([beta])
    ties = att = 0
    for sw in range(1, 5):
        cfg = b.download()["configs"][0].copy()
        b.record(True)
        b.run(1, or_per_metropolis=n_or, lanes_per_site=lanes, mode=mode, kernel=kernel, proposals=proposals)
        t, a, _ = check_pass(OH, cfg, b.fetch_record(-1), beta, "metro", seed=seed, sweep=sw, step=step)
        ties, att = ties + t, att + a
        for k in range(n_or):
            t, a, _ = check_pass(OH, cfg, b.fetch_record(k), beta, "or", seed=seed, sweep=sw, orpass=k)
            ties, att = ties + t, att + a
        post = b.download()
        np.testing.assert_array_equal(post["configs"][0], cfg)
        # FP64 recompute of the device state vs the oracle's total energy of the same spins
        E_dev = b.total_energy(0)
        E_or = OH.total_energy(post["configs"][0])
        assert abs(E_dev - E_or) <= 1e-10 * max(1.0, abs(E_or))
        # the running (FP32 dE, fixed-point summed) energy tracks the recompute
        assert abs(post["energies"][0] - E_or) <= 1e-5 * max(1.0, abs(E_or))
    assert ties <= max(1, att // 100)


# Every instance k_rep_colour<LMAX, P, NP, PF> of the replica-parallel kernel, forced
# through the run parameters: P replicas per thread, NP threads per item, PF prefetch
# (1 on, 2 off). Three replicas, so a P = 2 thread (G = 2) owns replicas 0 and 2 and
# replica 2 is its second lane; the recorded replica is that lane (P = 2) or the
# replica of the second thread of a site (P = 1).
REP_FORMS = [(P, NP, PF) for P in (1, 2) for NP in (1, 2) for PF in (1, 2)]


@pytest.mark.parametrize("name", ["bcc_body4", "fcc_l2_tri_zeeman", "bcc_l2_body3"])
@pytest.mark.parametrize("P,NP,PF", REP_FORMS, ids=[f"P{p}-NP{n}-PF{f}" for p, n, f in REP_FORMS])
def test_rep_colour_every_instance_replays(gpu, name, P, NP, PF):
    H, OH = build(name)
    gH = scemc.GPUTiledHamiltonian(H)
    R, step = 3, 0.6
    seeds = [0xA11CE + 17 * i for i in range(R)]
    betas = [1 / 0.05, 1 / 0.03, 1 / 0.08]
    rec = 2 if P == 2 else 1
    b = scemc.GPUBatch([gH], [R], [rand_cfg(H.n_sites, 40 + i) for i in range(R)], seeds, step)
    b.set_betas(betas)
    b.record_slot(0, rec)
    n_or = 2 if H.site_has_l1.any() else 0
    ties = att = 0
    for sw in range(1, 4):
        cfg = b.download()["configs"][rec].copy()
        b.record(True)
        b.run(1, or_per_metropolis=n_or, kernel=3, mode=1 + 2 * (sw == 3), proposals=1 + (sw % 2),
              rep_replicas=P, rep_threads_per_item=NP, rep_prefetch=PF)
        t, a, _ = check_pass(OH, cfg, b.fetch_record(-1), betas[rec], "metro", seed=seeds[rec], sweep=sw, step=step)
        ties, att = ties + t, att + a
        for k in range(n_or):
            t, a, _ = check_pass(OH, cfg, b.fetch_record(k), betas[rec], "or", seed=seeds[rec], sweep=sw, orpass=k)
            ties, att = ties + t, att + a
        post = b.download()
        np.testing.assert_array_equal(post["configs"][rec], cfg)
        E_or = OH.total_energy(post["configs"][rec])
        assert abs(b.total_energy(rec) - E_or) <= 1e-10 * max(1.0, abs(E_or))
        assert abs(post["energies"][rec] - E_or) <= 1e-5 * max(1.0, abs(E_or))
    assert ties <= max(1, att // 100)


@pytest.mark.parametrize("P,NP", [(1, 1), (1, 2), (2, 1), (2, 2)])
def test_rep_prefetch_changes_no_arithmetic(gpu, P, NP):
    """Prefetching the records and neighbour rows into L1 changes no arithmetic: the
    two forms give bitwise equal chains, overrelaxation included."""
    H, _ = build("fcc_l2_tri_zeeman")
    gH = scemc.GPUTiledHamiltonian(H)
    cfgs = [rand_cfg(H.n_sites, 60 + i) for i in range(3)]
    outs = []
    for PF in (1, 2):
        b = scemc.GPUBatch([gH], [3], cfgs, [5, 6, 7], 0.6)
        b.set_betas([1 / 0.05, 1 / 0.03, 1 / 0.08])
        b.run(5, or_per_metropolis=1, kernel=3, mode=1, rep_replicas=P, rep_threads_per_item=NP, rep_prefetch=PF)
        st = b.download()
        outs.append((np.stack(st["configs"]), st["energies"].copy(), st["counters"].copy()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][2], outs[1][2])


@pytest.mark.parametrize("P,NP", [(1, 1), (1, 2), (2, 1), (2, 2)])
def test_rep_persistent_equals_per_colour_launches(gpu, P, NP):
    """The persistent replica-parallel pass (one cooperative launch per pass, bounded
    grid barrier between colours, proposals precomputed inside it) gives chains bitwise
    equal to the per-colour launches of the same form, on a batch of two lattices."""
    w = models.config3_bcc_pt(sizes=(2, 3))
    Hs = [scemc.TiledHamiltonian(2, w.terms, dims=(s_, s_, s_)) for s_ in (2, 3)]
    gHs = [scemc.GPUTiledHamiltonian(H) for H in Hs]
    cfgs = [rand_cfg(H.n_sites, 50 + i) for i, H in enumerate(Hs) for _ in range(3)]
    betas = np.tile(1 / np.array([0.3e-3, 1e-3, 3e-3]), 2)
    outs = []
    for mode, prop in [(1, 1), (2, 1), (2, 2)]:
        b = scemc.GPUBatch(gHs, [3, 3], cfgs, [90 + i for i in range(6)], 0.6)
        b.set_betas(betas)
        b.run(6, kernel=3, mode=mode, proposals=prop, rep_replicas=P, rep_threads_per_item=NP, rep_prefetch=2,
              exchange=True, exchange_interval=1, phase_total=100)
        st = b.download()
        outs.append((np.concatenate([c.reshape(-1) for c in st["configs"]]), st["energies"].copy(),
                     st["counters"].copy(), st["slot_of_rung"].copy()))
    for o in outs[1:]:
        for x, y in zip(o, outs[0]):
            np.testing.assert_array_equal(x, y)


def test_rep_forms_refuse_bad_values(gpu):
    H, _ = build("bcc_body4")
    b = scemc.GPUBatch([scemc.GPUTiledHamiltonian(H)], [2], [rand_cfg(H.n_sites, 1)] * 2, [1, 2], 0.6)
    with pytest.raises(_lib.ScemcArgumentError):
        b.run(1, kernel=3, mode=1, rep_threads_per_item=3)
    with pytest.raises(_lib.ScemcArgumentError):
        b.run(1, kernel=3, mode=1, rep_prefetch=-1)
    with pytest.raises(_lib.ScemcArgumentError):
        b.record_slot(0, 2)
    with pytest.raises(_lib.ScemcArgumentError):
        b.record_slot(1, 0)


# The tensor-core replica pass (kernel 5) on every lmax-2 model with fast records: pair
# records only (biquadratic), l = 1 and l = 2 pairs (mixed), plaquette quads and
# Zeeman (bcc_l2_plaq_zeeman), l = 1 triangles (fcc), merged body-3 l <= 2 blocks
# (bcc_l2_body3). A warp owns 32 replicas of a site: R = 1 and 3 leave most rows of
# the tile empty; R = 32 records replica 25 (second 16-replica tile, row g + 8 of its
# fragment); R = 40 runs two chunks per site and records replica 37 (second chunk).
TC_MODELS = ["biquadratic_zeeman", "mixed", "bcc_l2_plaq_zeeman", "fcc_l2_tri_zeeman", "bcc_l2_body3"]
TC_SHAPES = [(1, 0), (3, 2), (32, 25), (40, 37)]


@pytest.mark.parametrize("name", TC_MODELS)
@pytest.mark.parametrize("R,rec", TC_SHAPES, ids=[f"R{r}-rec{k}" for r, k in TC_SHAPES])
def test_rep_tc_replays(gpu, name, R, rec):
    """Kernel 5 (pair records as mma.sync TF32 products, both operands split into a
    TF32 head and tail) replayed through the FP64 oracle: dE within the FP32 bar,
    identical decisions except ties, the proposals, the configuration after the
    compound sweep and the running energy, over Metropolis and overrelaxation passes
    with precomputed and inline proposals, per-colour launches and the graph."""
    H, OH = build(name)
    gH = scemc.GPUTiledHamiltonian(H)
    step = 0.6
    seeds = [0x7C0 + 13 * i for i in range(R)]
    betas = 1.0 / np.geomspace(0.02, 0.1, R)
    b = scemc.GPUBatch([gH], [R], [rand_cfg(H.n_sites, 300 + i) for i in range(R)], seeds, step)
    b.set_betas(betas)
    b.record_slot(0, rec)
    n_or = 2 if H.site_has_l1.any() else 0
    ties = att = 0
    for sw in range(1, 4):
        cfg = b.download()["configs"][rec].copy()
        b.record(True)
        b.run(1, or_per_metropolis=n_or, kernel=5, mode=1 + 2 * (sw == 3), proposals=1 + (sw % 2))
        t, a, _ = check_pass(OH, cfg, b.fetch_record(-1), betas[rec], "metro", seed=seeds[rec], sweep=sw, step=step)
        ties, att = ties + t, att + a
        for k in range(n_or):
            t, a, _ = check_pass(OH, cfg, b.fetch_record(k), betas[rec], "or", seed=seeds[rec], sweep=sw, orpass=k)
            ties, att = ties + t, att + a
        post = b.download()
        np.testing.assert_array_equal(post["configs"][rec], cfg)
        E_or = OH.total_energy(post["configs"][rec])
        assert abs(b.total_energy(rec) - E_or) <= 1e-10 * max(1.0, abs(E_or))
        assert abs(post["energies"][rec] - E_or) <= 1e-5 * max(1.0, abs(E_or))
    assert ties <= max(1, att // 100)


def test_rep_tc_refusals(gpu):
    """Kernel 5 needs lmax-2 fast tables, runs per-colour launches (mode 1 or 3) and
    plain proposals."""
    H, _ = build("bcc_body4")  # lmax 1
    b = scemc.GPUBatch([scemc.GPUTiledHamiltonian(H)], [2], [rand_cfg(H.n_sites, 1)] * 2, [1, 2], 0.6)
    with pytest.raises(_lib.ScemcArgumentError):
        b.run(1, kernel=5, mode=1)
    H2, _ = build("fcc_l2_tri_zeeman")
    b2 = scemc.GPUBatch([scemc.GPUTiledHamiltonian(H2)], [2], [rand_cfg(H2.n_sites, 1)] * 2, [1, 2], 0.6)
    for mode in (2, 4):
        with pytest.raises(_lib.ScemcArgumentError):
            b2.run(1, kernel=5, mode=mode)
    b2.run(2, kernel=5, mode=3, or_per_metropolis=1)


@pytest.mark.parametrize("kernel,recs", [(3, (0, 17)), (5, (0, 25))])
def test_fcc64_32_rungs_replays_at_full_size(gpu, kernel, recs):
    """The large frustrated configuration at its own size (fcc 64^3 x 4 sites, 32
    rungs, kT geometric in [0.05, 2.0] meV). Kernel 3 runs the form the library picks
    by itself: its colours fill many waves, so k_rep_colour runs with two replicas per
    thread, one thread per item and no prefetch; rung 0 (the first lane of a thread)
    and rung 17 (the second lane of thread 1) are recorded. Kernel 5 (the tensor-core
    pass) records rung 0 and rung 25 (second 16-replica tile, fragment row g + 8).
    Each recorded rung is replayed over a Metropolis and an overrelaxation pass
    through the FP64 oracle (dE and the decisions at every site, the proposals at
    3000 sampled sites)."""
    w = models.config5_fcc(n=64, replicas=32)
    H = w.hamiltonians()[0]
    OH = O.OracleHamiltonian(4, w.terms, (64, 64, 64), magmoms=w.magmoms, field=w.field)
    gH = scemc.GPUTiledHamiltonian(H)
    R, step = 32, 0.6
    seeds = [0x5EED0 + 3 * r for r in range(R)]
    betas = 1.0 / w.kts
    base = rand_cfg(H.n_sites, 77)
    cfgs = [np.roll(base, 7 * r, axis=0) for r in range(R)]
    b = scemc.GPUBatch([gH], [R], cfgs, seeds, step)
    b.set_betas(betas)
    ties = att = 0
    for sw, rec in zip((1, 2), recs):
        b.record_slot(0, rec)
        cfg = b.download()["configs"][rec].copy()
        b.record(True)
        b.run(1, or_per_metropolis=1, kernel=kernel, mode=1)
        t, a, _ = check_pass(OH, cfg, b.fetch_record(-1), betas[rec], "metro", seed=seeds[rec], sweep=sw,
                             step=step, sample=3000)
        ties, att = ties + t, att + a
        t, a, _ = check_pass(OH, cfg, b.fetch_record(0), betas[rec], "or", seed=seeds[rec], sweep=sw, orpass=0,
                             sample=3000)
        ties, att = ties + t, att + a
        np.testing.assert_array_equal(b.download()["configs"][rec], cfg)
        E_or = OH.total_energy(cfg)
        assert abs(b.total_energy(rec) - E_or) <= 1e-10 * max(1.0, abs(E_or))
    assert att > 3 * H.n_sites
    assert ties <= max(1, att // 100)


def test_step_adaptation_follows_the_oracle(gpu):
    """Device step adaptation (k_tail) against the oracle's _adapt_step! law
    (updates.jl:296-305): every adapt_interval sweeps of a thermalisation phase, the
    step of each rung becomes clamp(step exp((a - target) / 2), 1e-3, pi) with a the
    Metropolis acceptance of that window. The windows are read back from the counters
    and the whole per-rung step trajectory is recomputed by the oracle."""
    H, _ = build("bcc_l2_plaq_zeeman")
    gH = scemc.GPUTiledHamiltonian(H)
    R, interval, target = 4, 10, 0.5
    kts = np.array([0.02, 0.2, 2.0, 20.0]) * 1e-3  # from near-frozen to hot: the step shrinks and grows
    steps0 = np.array([0.6, 0.6, 2.0, 3.0])
    b = scemc.GPUBatch([gH], [R], [rand_cfg(H.n_sites, 90 + r) for r in range(R)], [11, 12, 13, 14], steps0)
    b.set_betas(1.0 / kts)
    expect = steps0.copy()
    hit_clamp = False
    for win in range(12):
        before = b.download()["counters"].copy()
        b.run(interval, adapt_interval=interval, adapt_target=target, phase_done=win * interval,
              phase_total=12 * interval, kernel=1, mode=2)
        st = b.download()
        d = st["counters"] - before
        for r in range(R):
            expect[r] = O.adapt_step(expect[r], d[r, 0], d[r, 1], target)
            hit_clamp |= expect[r] in (1e-3, math.pi)
        np.testing.assert_allclose(st["steps"], expect, rtol=1e-14, atol=0)
    assert hit_clamp or np.ptp(expect) > 0.5


def test_fast_kernel_is_launch_shape_independent(gpu):
    """The fast kernel fixes its lane count by lmax and reduces dE with a fixed
    butterfly: per-colour vs persistent launches and precomputed vs inline proposals
    give bitwise-identical chains, overrelaxation included. The replica-parallel
    kernel gives the same chains with one or two replicas per thread."""
    H, _ = build("bcc_l2_plaq_zeeman")
    gH = scemc.GPUTiledHamiltonian(H)
    cfg = rand_cfg(H.n_sites, 3)
    # kernel 3 also with one and two replicas per thread (three replicas: the second
    # thread of a site carries one unused slot when it owns two)
    for kernel, R, forms in [(2, 2, [(1, 1, 0), (1, 2, 0), (2, 1, 0), (2, 2, 0), (3, 1, 0), (3, 2, 0), (4, 1, 0),
                                     (4, 2, 0)]),
                             (3, 3, [(1, 1, 0), (1, 2, 1), (3, 1, 2), (3, 2, 1), (1, 1, 2), (3, 1, 0)])]:
        outs = []
        for mode, prop, rr in forms:
            b = scemc.GPUBatch([gH], [R], [cfg] * R, [9, 10, 11][:R], 0.6)
            b.set_betas([1 / 0.002, 1 / 0.01, 1 / 0.005][:R])
            b.run(6, or_per_metropolis=1, mode=mode, proposals=prop, kernel=kernel, rep_replicas=rr)
            st = b.download()
            outs.append((np.stack(st["configs"]), st["energies"].copy(), st["counters"].copy()))
        for o in outs[1:]:
            assert np.array_equal(o[0], outs[0][0]) and np.array_equal(o[1], outs[0][1])
            assert np.array_equal(o[2], outs[0][2])


def test_cluster_kernel_equals_row_parallel_kernel(gpu):
    """The chain-resident cluster kernel (kernel 4: one thread-block cluster per
    replica slot, the replica's spins in every CTA's shared memory, colours separated
    by the cluster barrier) runs the row-parallel arithmetic: its chains are bitwise
    those of the row-parallel kernel, for several replicas and for a batch of two
    lattices of different sizes, with per-sweep launches and in a CUDA graph, with
    precomputed and inline proposals, overrelaxation included."""
    w = models.config2_bcc_l2(n=3)
    Hs = [scemc.TiledHamiltonian(2, w.terms, dims=(d, d, d), magmoms=w.magmoms, field=w.field) for d in (3, 4)]
    gHs = [scemc.GPUTiledHamiltonian(H) for H in Hs]
    cfgs = [rand_cfg(H.n_sites, 30 + i) for i, H in enumerate(Hs) for _ in range(3)]
    betas = np.tile(1 / np.array([0.2e-3, 1e-3, 2e-3]), 2)
    outs = []
    for kernel, mode, prop in [(2, 1, 1), (4, 1, 1), (4, 1, 2), (4, 3, 1), (4, 3, 2)]:
        b = scemc.GPUBatch(gHs, [3, 3], cfgs, [70 + i for i in range(6)], 0.6)
        b.set_betas(betas)
        b.run(7, or_per_metropolis=2, kernel=kernel, mode=mode, proposals=prop)
        st = b.download()
        outs.append((np.concatenate([c.reshape(-1) for c in st["configs"]]), st["energies"].copy(),
                     st["counters"].copy()))
    for o in outs[1:]:
        np.testing.assert_array_equal(o[0], outs[0][0])
        np.testing.assert_array_equal(o[1], outs[0][1])
        np.testing.assert_array_equal(o[2], outs[0][2])


def test_cluster_kernel_refusals(gpu):
    H, _ = build("bcc_l2_plaq_zeeman")
    b = scemc.GPUBatch([scemc.GPUTiledHamiltonian(H)], [1], [rand_cfg(H.n_sites, 1)], [1], 0.6)
    with pytest.raises(_lib.ScemcArgumentError):
        b.run(1, kernel=4, mode=2)
    Hm, _ = build("high_l")  # no fast tables (l = 3 and 4 members)
    bm = scemc.GPUBatch([scemc.GPUTiledHamiltonian(Hm)], [1], [rand_cfg(Hm.n_sites, 1)], [1], 0.6)
    with pytest.raises(_lib.ScemcArgumentError):
        bm.run(1, kernel=4)
    w = models.config2_bcc_l2(n=24)  # 27,648 sites x 16 bytes: more than one block's shared memory
    Hb = w.hamiltonians()[0]
    bb = scemc.GPUBatch([scemc.GPUTiledHamiltonian(Hb)], [1], [rand_cfg(Hb.n_sites, 1)], [1], 0.6)
    with pytest.raises(_lib.ScemcArgumentError, match="shared memory"):
        bb.run(1, kernel=4)


def test_autotune_keeps_a_valid_launch_form(gpu):
    H, _ = build("bcc_l2_plaq_zeeman")
    gH = scemc.GPUTiledHamiltonian(H)
    b = scemc.GPUBatch([gH], [3], [rand_cfg(H.n_sites, i) for i in range(3)], [1, 2, 3], 0.6)
    b.set_betas([1 / 0.002, 1 / 0.004, 1 / 0.008])
    t = b.autotune(or_per_metropolis=1, sweeps_per_trial=3)
    assert t["mode"] in (2, 3, 4) and t["proposals"] in (1, 2) and t["kernel"] in (2, 3, 4, 5) and t["ms_per_sweep"] > 0
    if t["kernel"] in (4, 5):
        assert t["mode"] == 3
    if t["kernel"] == 3:
        assert t["mode"] in (2, 3)
    before = b.download()["counters"].copy()
    b.run(4, or_per_metropolis=1)  # mode 0 now uses the tuned form
    after = b.download()["counters"]
    assert np.all(after[:, 1] - before[:, 1] == 4 * H.n_active)
    for r in range(3):
        st = b.download()
        assert abs(st["energies"][r] - b.total_energy(r)) <= 1e-5 * max(1.0, abs(st["energies"][r]))


def test_fast_kernel_refused_where_it_does_not_apply(gpu):
    H, _ = build("high_l")
    gH = scemc.GPUTiledHamiltonian(H)
    b = scemc.GPUBatch([gH], [1], [rand_cfg(H.n_sites, 1)], [1], 0.6)
    with pytest.raises(_lib.ScemcArgumentError):
        b.run(1, kernel=2)
    with pytest.raises(_lib.ScemcArgumentError):
        b.run(1, kernel=3)
    b.run(1, kernel=0)  # auto falls back to the generic record walk
    H2, _ = build("bcc_l2_plaq_zeeman")
    b2 = scemc.GPUBatch([scemc.GPUTiledHamiltonian(H2)], [1], [rand_cfg(H2.n_sites, 1)], [1], 0.6)
    b2.run(1, kernel=3, mode=2)  # the replica-parallel kernel's persistent form


def test_proposal_stream_is_the_reference_stream(gpu):
    """A single chain's Metropolis draws are the reference's keyed stream (tag 0)."""
    H, OH = build("chain")
    gH = scemc.GPUTiledHamiltonian(H)
    b = scemc.GPUBatch([gH], [1], [rand_cfg(H.n_sites, 1)], [0xBEEF], 0.6)
    b.set_betas([1.0])
    b.record(True)
    b.run(1, lanes_per_site=1, mode=1)
    prop, u, _, flag = b.fetch_record(-1)
    for s in range(H.n_sites):
        b0 = O.philox_block(0xBEEF, s + 1, 1, 0)
        assert u[s] == O.philox_uniform(b0[2], b0[3])


def test_energy_recompute_and_drift(gpu):
    H, OH = build("biquadratic")
    gH = scemc.GPUTiledHamiltonian(H)
    cfg = rand_cfg(H.n_sites, 7)
    gst = scemc.GPUChainState(gH, cfg, seed=0xC0FFEE)
    E0 = OH.total_energy(np.asarray(cfg, np.float32).astype(np.float64))
    assert abs(gst.energy - E0) <= 1e-10 * max(1, abs(E0))
    st = scemc.ChainState(cfg, gst.energy)
    scemc.gpu_run_sweeps(gst, gH, st, 1 / 0.05, 200, renorm_interval=0)
    E = OH.total_energy(st.config)
    drift = abs(gst.energy - E)
    assert drift <= 1e-6 * max(1.0, abs(E)), drift
    d = gst.renormalize()
    assert d == pytest.approx(drift, rel=1e-3, abs=1e-15)
    assert abs(gst.energy - OH.total_energy(scemc.to_host(st, gst).config)) <= 1e-10 * max(1.0, abs(E))


def test_repeat_identity_lanes_and_modes(gpu):
    """Bitwise repeatability for a fixed (seed, lanes, launch form); the launch form
    does not change the chain; other lane counts only reorder FP32 sums, so a
    Metropolis-only chain stays on the same trajectory (overrelaxation is a
    chaotic deterministic map, so it is compared through the replay gates only)."""
    H, _ = build("bcc_l2_plaq_zeeman")
    gH = scemc.GPUTiledHamiltonian(H)
    cfg = rand_cfg(H.n_sites, 3)

    def run(lanes, mode, seed, n_or):
        b = scemc.GPUBatch([gH], [1], [cfg], [seed], 0.6)
        b.set_betas([1 / 0.002])
        b.run(6, or_per_metropolis=n_or, lanes_per_site=lanes, mode=mode, kernel=1)
        st = b.download()
        return st["configs"][0], st["energies"][0], st["counters"][0].copy()

    a, b_, c = run(4, 2, 9, 1), run(4, 2, 9, 1), run(4, 1, 9, 1)
    assert np.array_equal(a[0], b_[0]) and a[1] == b_[1] and np.array_equal(a[2], b_[2])
    assert np.array_equal(a[0], c[0]) and a[1] == c[1]
    m = [run(g, 2, 9, 0) for g in (4, 1, 32)]
    for k in (1, 2):
        assert np.max(np.abs(m[0][0] - m[k][0])) < 1e-5
        assert np.array_equal(m[0][2], m[k][2])
    assert not np.array_equal(run(4, 2, 10, 1)[0], a[0])


def test_inactive_sites_frozen(gpu):
    H, _ = build("dimer")
    gH = scemc.GPUTiledHamiltonian(H)
    cfg = rand_cfg(H.n_sites, 7)
    gst = scemc.GPUChainState(gH, cfg, seed=1)
    st = scemc.ChainState(cfg, gst.energy)
    scemc.gpu_run_sweeps(gst, gH, st, 1 / 0.05, 50, renorm_interval=20)
    np.testing.assert_array_equal(st.config[2:], cfg[2:].astype(np.float32).astype(np.float64))


def test_batch_of_uneven_lattices_equals_single_chains(gpu):
    """Chains of different supercells in one batch follow exactly the trajectories
    they follow alone (keyed RNG, per-item independence)."""
    w = models.config3_bcc_pt(sizes=(2, 3))
    Hs = [scemc.TiledHamiltonian(2, w.terms, dims=(s, s, s)) for s in (2, 3)]
    gHs = [scemc.GPUTiledHamiltonian(H) for H in Hs]
    cfgs = [rand_cfg(H.n_sites, 20 + i) for i, H in enumerate(Hs) for _ in range(3)]
    seeds = [100 + i for i in range(6)]
    betas = np.tile(1 / np.array([0.3e-3, 1e-3, 3e-3]), 2)
    b = scemc.GPUBatch(gHs, [3, 3], cfgs, seeds, 0.6)
    b.set_betas(betas)
    b.run(5, lanes_per_site=2, mode=2)
    got = b.download()
    for i in range(6):
        gH = gHs[i // 3]
        one = scemc.GPUBatch([gH], [1], [cfgs[i]], [seeds[i]], 0.6)
        one.set_betas([betas[i]])
        one.run(5, lanes_per_site=2, mode=2)
        st = one.download()
        np.testing.assert_array_equal(got["configs"][i], st["configs"][0])
        assert got["energies"][i] == st["energies"][0]


def test_swap_payload_and_roundtrip(gpu):
    H, _ = build("biquadratic")
    gH = scemc.GPUTiledHamiltonian(H)
    a = scemc.GPUChainState(gH, rand_cfg(H.n_sites, 1), seed=1)
    b = scemc.GPUChainState(gH, rand_cfg(H.n_sites, 2), seed=2)
    scemc.gpu_metropolis_sweep(a, gH, 20.0)
    sa, sb = scemc.ChainState(None, 0), scemc.ChainState(None, 0)
    scemc.to_host(sa, a), scemc.to_host(sb, b)
    ca, cb = a.counters().copy(), b.counters().copy()
    ia, ib = a.sweep_index, b.sweep_index
    scemc.swap_payload(a, b)
    ta, tb = scemc.ChainState(None, 0), scemc.ChainState(None, 0)
    scemc.to_host(ta, a), scemc.to_host(tb, b)
    np.testing.assert_array_equal(ta.config, sb.config)
    np.testing.assert_array_equal(tb.config, sa.config)
    assert ta.energy == sb.energy and tb.energy == sa.energy
    assert np.array_equal(a.counters(), ca) and np.array_equal(b.counters(), cb)
    assert (a.sweep_index, b.sweep_index) == (ia, ib)
    # upload/download round trip keeps FP32 values exactly
    scemc.from_host(a, sa)
    scemc.to_host(ta, a)
    np.testing.assert_array_equal(ta.config, sa.config)


def test_batch_payload_round_trip_and_guard(gpu):
    """Uploads and downloads of a batch of uneven tables: the device rounds and
    interleaves the host payload exactly like an FP32 cast, a download into a
    pinned buffer equals the default one, and a non-finite spin is reported by its
    replica and column with the device state left as it was."""
    Hs = [build("bcc_body4")[0], scemc.TiledHamiltonian(2, models.config4_bcc_body4().terms, dims=(2, 3, 4))]
    gHs = [scemc.GPUTiledHamiltonian(h) for h in Hs]
    reps = [3, 2]
    cfgs = [rand_cfg(h.n_sites, 40 + 7 * i + r) for i, h in enumerate(Hs) for r in range(reps[i])]
    b = scemc.GPUBatch(gHs, reps, cfgs, list(range(1, 6)), 0.5, energies=np.zeros(5))  # no renormalisation
    got = b.download()
    for c, g in zip(cfgs, got["configs"]):
        np.testing.assert_array_equal(g, c.astype(np.float32).astype(np.float64))
    en = np.arange(5, dtype=np.float64) * 0.25 - 1.0
    new = [rand_cfg(h.n_sites, 90 + 3 * i + r) for i, h in enumerate(Hs) for r in range(reps[i])]
    b.upload(np.concatenate([c.reshape(-1) for c in new]), en)
    with scemc.PinnedHost(3 * b.n_sites_total) as pin:
        a = b.download(out=pin.array)
        b.upload(pin.array, en)  # a pinned payload round-trips unchanged
        a = {k: (v.copy() if isinstance(v, np.ndarray) else [c.copy() for c in v]) for k, v in
             b.download(out=pin.array).items()}
    d = b.download()
    for c, x, y in zip(new, a["configs"], d["configs"]):
        np.testing.assert_array_equal(x, c.astype(np.float32).astype(np.float64))
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a["energies"], en)
    for k in ("slot_of_rung", "counters", "swaps", "steps", "max_drift"):
        np.testing.assert_array_equal(a[k], d[k])
    bad = np.concatenate([c.reshape(-1) for c in cfgs])
    off = 3 * Hs[0].n_sites * reps[0] + 3 * Hs[1].n_sites  # table 2, replica 2
    bad[off + 3 * 4 + 1] = np.inf  # its column 5
    with pytest.raises(scemc.ScemcError, match="column 5 of replica 2"):
        b.upload(bad, en + 1.0)
    after = b.download()
    for c, x in zip(new, after["configs"]):
        np.testing.assert_array_equal(x, c.astype(np.float32).astype(np.float64))
    np.testing.assert_array_equal(after["energies"], en)
    with pytest.raises(_lib.ScemcArgumentError):
        b.upload(np.concatenate([c.reshape(-1) for c in cfgs]), np.full(5, np.nan))
    with pytest.raises(ValueError):
        b.download(out=np.zeros(7))


def test_guards(gpu):
    H, _ = build("chain")
    gH = scemc.GPUTiledHamiltonian(H)
    gst = scemc.GPUChainState(gH, rand_cfg(H.n_sites, 1), seed=1)
    with pytest.raises(ValueError):
        scemc.gpu_metropolis_sweep(gst, gH, 1.0, workgroupsize=3)
    with pytest.raises(_lib.ScemcArgumentError):
        _lib.check(_lib.lib().scemc_metropolis_sweep(gst.h, gH.h, 1.0, 3, None))
    bad = np.full((H.n_sites, 3), np.nan)
    with pytest.raises(scemc.ScemcError):
        scemc.GPUChainState(gH, bad, seed=1, energy=0.0)
    # lmax > 6 refused at table upload (gpu_hamiltonian.jl:67-68)
    f = np.zeros((15, 3))
    f[0, 0] = 1.0
    H7 = scemc.TiledHamiltonian(1, [scemc.MultipoleTerm(1.0, [1, 1], [(0, 0, 0), (1, 0, 0)], [7, 1], f)],
                                dims=(3, 1, 1))
    with pytest.raises(ValueError):
        scemc.GPUTiledHamiltonian(H7)
    d = H7.desc()
    h = _lib.C.c_void_p()
    assert _lib.lib().scemc_tables_create(_lib.C.byref(d), _lib.C.byref(h)) == _lib.ERR_UNSUPPORTED
    # a corrupted table is refused, not uploaded
    Hc, _ = build("biquadratic")
    Hc.site_prog = Hc.site_prog.copy()
    Hc.site_prog[0] += 1
    with pytest.raises(_lib.ScemcArgumentError):
        scemc.GPUTiledHamiltonian(Hc)


def test_barrier_timeout_is_bounded(gpu):
    """Failure detection: a grid barrier that can never complete gives up after its
    bound and reports SCEMC_ERR_TIMEOUT; the context stays usable."""
    assert _lib.lib().scemc_selftest_barrier_timeout(50_000_000) == _lib.ERR_TIMEOUT
    H, _ = build("chain")
    gH = scemc.GPUTiledHamiltonian(H)
    gst = scemc.GPUChainState(gH, rand_cfg(H.n_sites, 1), seed=1)
    assert scemc.gpu_metropolis_sweep(gst, gH, 1.0) >= 0


# -- statistics -------------------------------------------------------------------------
def langevin(x):
    return 1.0 / math.tanh(x) - 1.0 / x


def test_dimer_langevin_and_pt_marginals(gpu):
    """<E> = J L(beta|J|) at every rung of an exchanging 3-rung ladder (test_gpu_pt.jl:13-42)."""
    J = -0.02
    gH = scemc.GPUTiledHamiltonian(models.dimer(J=J))
    kts = abs(J) * np.array([0.3, 0.6, 1.2])
    r = scemc.gpu_run_pt(gH, kT=kts, sweeps_therm=500, sweeps_measure=20000, measure_interval=5,
                         exchange_interval=10, seed=31)
    for p, kt in zip(r.points, kts):
        exact = J * langevin(abs(J) / kt)
        E, err = p.stats["energy"].mean[0], p.stats["energy"].err[0]
        assert abs(E - exact) < 5 * err + 1e-3 * abs(J)
        assert abs(E - exact) < 0.04 * abs(J)
        np.testing.assert_array_equal(p.stats["sublattice_m"].mean[6:12], np.zeros(6))
    assert len(r.swap_acceptance) == 2 and np.all((r.swap_acceptance > 0) & (r.swap_acceptance <= 1))


def test_exchange_rate_limits(gpu):
    """test_gpu_pt.jl:44-60: a degenerate ladder always swaps; a wide one rarely, and
    the rung energies are ordered."""
    gH = scemc.GPUTiledHamiltonian(models.dimer())
    r = scemc.gpu_run_pt(gH, kT=[0.049999, 0.05], sweeps_therm=100, sweeps_measure=400, exchange_interval=5,
                         seed=1)
    assert r.swap_acceptance[0] > 0.95
    H = scemc.TiledHamiltonian(1, models.chain_terms(-0.05), dims=(4, 4, 2))
    gH2 = scemc.GPUTiledHamiltonian(H)
    r2 = scemc.gpu_run_pt(gH2, kT=[0.002, 0.2], sweeps_therm=200, sweeps_measure=1000, exchange_interval=5, seed=2)
    assert r2.swap_acceptance[0] < 0.2
    Es = [p.stats["energy"].mean[0] for p in r2.points]
    assert Es[0] < Es[1]


def test_single_moment_in_a_field(gpu):
    """<e_z> = -L(beta h) for h e_z, and a Zeeman-only moment: test_gpu.jl:458-484."""
    c0 = 0.3
    h = c0 * scemc.N1
    gH = scemc.GPUTiledHamiltonian(scemc.TiledHamiltonian(1, models.single_site_terms(c0)))
    r = scemc.gpu_run_pt(gH, kT=[h / 1.0, h / 2.0], exchange=False, sweeps_therm=500, sweeps_measure=40000,
                         measure_interval=2, step=1.2, seed=202)
    for p, bh in zip(r.points, (1.0, 2.0)):
        assert p.stats["energy"].mean[0] / h == pytest.approx(-langevin(bh), abs=0.03)


def compare_stats(a, b, names, n_sigma=3.0, comps=None):
    """Agreement within combined error bars; returns the list of z-scores."""
    zs, report = [], []
    for n in names:
        ma, ea = np.asarray(a[n][0]), np.asarray(a[n][1])
        mb, eb = np.asarray(b[n][0]), np.asarray(b[n][1])
        if comps and n in comps:
            ma, ea, mb, eb = ma[comps[n]], ea[comps[n]], mb[comps[n]], eb[comps[n]]
        z = np.abs(ma - mb) / np.sqrt(ea ** 2 + eb ** 2 + 1e-300)
        zs += list(z)
        report.append((n, ma, mb, ea, eb, z))
    for r in report:
        assert np.all(r[5] < n_sigma), report
    return zs


def as_tuple_stats(stats):
    return {k: (v.mean, v.err) for k, v in stats.items()}


def test_sc_J1J2_statistics_match_cpu_run_mc(gpu):
    """Config-1 physics (sc 8^3 J1/J2, kT 0.5 meV): E, C, |m|, chi and U of the device
    chain agree with the oracle's run_mc within their error bars. (The vector m of
    an isotropic ferromagnet only diffuses in direction, so its components are not
    compared here; the field-bearing model below compares sublattice vectors.)"""
    w = models.config1_sc()
    H = w.hamiltonians()[0]
    OH = O.OracleHamiltonian(1, w.terms, (8, 8, 8))
    kT = float(w.kts[0])
    gH = scemc.GPUTiledHamiltonian(H)
    r = scemc.gpu_run_pt(gH, kT=[kT], exchange=False, sweeps_therm=2000, sweeps_measure=20000, seed=1)
    ch = O.OracleChain(OH, models.random_config(H.n_sites, 11), seed=11)
    ost = ch.run_mc(kT, 2000, 20000)
    names = ["energy", "specific_heat", "absm", "susceptibility", "binder"]
    zs = compare_stats(as_tuple_stats(r.points[0].stats), ost, names, n_sigma=4.0)
    assert sum(z > 2.0 for z in zs) <= 1, zs
    assert abs(r.points[0].acceptance_metropolis - ost["acceptance_metropolis"]) < 0.02


def test_bcc_multipole_or_statistics_match_cpu(gpu):
    """Metropolis + overrelaxation on the l<=2 + plaquette + Zeeman model (config-2
    shape, 4^3) at kT = 4 meV, where it equilibrates quickly: energy, |m| and the
    field-aligned sublattice magnetisation agree with the oracle's run_mc."""
    w = models.config2_bcc_l2(n=4)
    H = w.hamiltonians()[0]
    OH = O.OracleHamiltonian(2, w.terms, (4, 4, 4), magmoms=w.magmoms, field=w.field)
    kT = 4.0e-3
    gH = scemc.GPUTiledHamiltonian(H)
    r = scemc.gpu_run_pt(gH, kT=[kT], exchange=False, sweeps_therm=2000, sweeps_measure=20000, or_per_metropolis=1,
                         seed=2)
    ch = O.OracleChain(OH, models.random_config(H.n_sites, 2), seed=2)
    ost = ch.run_mc(kT, 2000, 20000, n_or=1)
    p = r.points[0]
    assert 0.0 < p.acceptance_or < 1.0
    assert abs(p.acceptance_or - ost["acceptance_or"]) < 0.02
    zs = compare_stats(as_tuple_stats(p.stats), ost, ["energy", "specific_heat", "absm", "m2", "sublattice_m"],
                       n_sigma=4.0, comps={"sublattice_m": [2, 5]})
    assert sum(z > 2.0 for z in zs) <= 1, zs


def test_pt_energies_match_cpu_run_pt(gpu):
    w = models.config3_bcc_pt()
    dims = (3, 3, 3)
    H = scemc.TiledHamiltonian(2, w.terms, dims=dims)
    OH = O.OracleHamiltonian(2, w.terms, dims)
    kts = np.geomspace(1.0, 6.0, 4) * 1e-3
    gH = scemc.GPUTiledHamiltonian(H)
    r = scemc.gpu_run_pt(gH, kT=kts, exchange_interval=1, sweeps_therm=2000, sweeps_measure=20000, seed=3)
    chains = [O.OracleChain(OH, models.random_config(H.n_sites, 30 + i), seed=300 + i) for i in range(4)]
    pts, swaps = O.run_pt(OH, chains, kts, 2000, 20000, exchange_interval=1)
    zs = []
    for p, q in zip(r.points, pts):
        zs += compare_stats(as_tuple_stats(p.stats), q, ["energy", "absm"], n_sigma=4.0)
    assert sum(z > 2.0 for z in zs) <= 2, zs
    np.testing.assert_allclose(r.swap_acceptance, swaps, atol=0.05)


def test_launch_count_matches_the_launch_form(gpu):
    """scemc_batch_launches counts every kernel the batch enqueues: per compound sweep
    of per-colour launches, one precompute launch plus one launch per colour and pass
    plus the tail; a replayed graph adds the same kernel nodes."""
    H, _ = build("bcc_l2_plaq_zeeman")
    gH = scemc.GPUTiledHamiltonian(H)
    b = scemc.GPUBatch([gH], [2], [rand_cfg(H.n_sites, 1), rand_cfg(H.n_sites, 2)], [1, 2], 0.6)
    per_sweep = 1 + 2 * H.n_colors + 1
    for kernel, mode in [(2, 1), (2, 3), (3, 1), (3, 3), (5, 1), (5, 3)]:
        b.run(1, or_per_metropolis=1, mode=mode, kernel=kernel, proposals=1)  # graph capture, if any
        n0 = b.launches()
        b.run(3, or_per_metropolis=1, mode=mode, kernel=kernel, proposals=1)
        assert b.launches() - n0 == 3 * per_sweep, (kernel, mode)
    for mode in (2, 4):  # one persistent launch per pass + tail
        n0 = b.launches()
        b.run(2, or_per_metropolis=1, mode=mode, kernel=2, proposals=2)
        assert b.launches() - n0 == 2 * 3


@pytest.mark.parametrize("name", ["dimer_zeeman", "biquadratic_zeeman", "mixed", "high_l", "fourbody",
                                  "bcc_l2_plaq_zeeman", "fcc_l2_tri_zeeman"])
def test_energy_gradient_matches_oracle(gpu, name):
    """The all-site tangent gradient (gpu_energy_gradient!) against the FP64 oracle on
    the same FP32-rounded spins: FP32 coefficients, FP64 gradient rows."""
    H, OH = build(name)
    gH = scemc.GPUTiledHamiltonian(H)
    cfgs = np.stack([rand_cfg(H.n_sites, 60 + r) for r in range(3)])
    G = scemc.gpu_energy_gradient(gH, cfgs)
    assert G.shape == cfgs.shape
    for r in range(3):
        ref = OH.energy_gradient(cfgs[r].astype(np.float32).astype(np.float64))
        tol = 2e-5 * np.abs(ref).max() + 1e-30
        assert np.abs(G[r] - ref).max() <= tol, (name, r, np.abs(G[r] - ref).max(), tol)
    np.testing.assert_allclose(scemc.gpu_energy_gradient(gH, cfgs[1]), G[1])
