"""Pins the FP64 oracle before it is trusted as the checker.

Known answers from the reference's own tests (tests/golden/philox_kat.json,
extracted from test/unit/test_gpu.jl:49-71), analytic tesseral rows, exactness
identities of the energy contract (test/unit/test_energy.jl), the colouring
contract (test/unit/test_parallel.jl:7-24) and closed-form statistics
(test/unit/test_metropolis.jl:10-49). CPU only.
"""
import json
import math
import pathlib
from fractions import Fraction

import numpy as np
import pytest

import oracle as O
import scemc
from scemc import models

GOLD = json.loads((pathlib.Path(__file__).parent / "golden" / "philox_kat.json").read_text())


def langevin(x):
    return 1.0 / math.tanh(x) - 1.0 / x


# -- keyed RNG -----------------------------------------------------------------
def test_philox_known_answers():
    assert len(GOLD["philox4x32_10"]) == 3
    for kat in GOLD["philox4x32_10"]:
        assert O.philox4x32(kat["ctr"], kat["key"]) == tuple(kat["out"])


def test_uniform_open_interval_and_streams():
    lo_w, hi_w = GOLD["uniform_edge_words"]
    assert 0.0 < O.philox_uniform(*lo_w)
    assert O.philox_uniform(*hi_w) < 1.0
    assert O.philox_uniform(0, 0) == 2.0 ** -53
    blk = O.philox_block(1, 3, 5, 0)
    assert blk != O.philox_block(2, 3, 5, 0)
    assert blk != O.philox_block(1, 4, 5, 0)
    assert blk != O.philox_block(1, 3, 6, 0)
    assert blk != O.philox_block(1, 3, 5, 1)
    assert blk != O.philox_block(1, 3, 5, 0, tag=1)
    assert blk == O.philox_block(1, 3, 5, 0)
    n1, n2 = O.philox_normal2(blk)
    assert math.isfinite(n1) and math.isfinite(n2)
    # key = (lo32(seed), hi32(seed)), ctr = (site, sweep, slot, 0)
    seed = 0x299F31D0A4093822
    assert O.philox_block(seed, 0x243F6A88 - (1 << 32), 0x85A308D3 - (1 << 32), 0x13198A2E, 0x03707344) == \
        O.philox4x32((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0))


def test_proposal_reads_named_slots():
    """Value pin of the proposal's slot map (test_gpu.jl:219-251)."""
    seed, e, step = 0xBEEF, np.array([0.0, 0.0, 1.0]), 0.6
    nflip = 0
    for site in range(1, 25):
        for sw in range(1, 5):
            b0 = O.philox_block(seed, site, sw, 0)
            u_flip, u_acc = O.philox_uniform(b0[0], b0[1]), O.philox_uniform(b0[2], b0[3])
            e2, ua = O.keyed_proposal(seed, site, sw, e, step)
            assert ua == u_acc
            if u_flip < 0.2:
                nflip += 1
                assert np.array_equal(e2, -e)
            else:
                n1, n2 = O.philox_normal2(O.philox_block(seed, site, sw, 1))
                n3, n4 = O.philox_normal2(O.philox_block(seed, site, sw, 2))
                nn = math.sqrt((n1 * n1 + n2 * n2) + n3 * n3)
                ref = O.rotate(e, np.array([n1 / nn, n2 / nn, n3 / nn]), step * n4)
                assert np.array_equal(e2, ref)
    assert 0 < nflip < 96


# -- tesseral rows ---------------------------------------------------------------
def _dirs(n=400, seed=2026):
    rng = np.random.default_rng(seed)
    d = [np.array(v, float) for v in [(0, 0, 1), (0, 0, -1), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0)]]
    for k in range(12):
        d.append(np.array([math.cos(k * math.pi / 6), math.sin(k * math.pi / 6), 0.0]))
    v = rng.standard_normal((n, 3))
    d += list(v / np.linalg.norm(v, axis=1, keepdims=True))
    return d


def test_zlm_low_l_closed_forms():
    N1 = math.sqrt(3 / (4 * math.pi))
    for u in _dirs():
        x, y, z = u
        row = O.zlm_row(2, u)
        assert row[0] == pytest.approx(1 / math.sqrt(4 * math.pi), abs=1e-15)
        np.testing.assert_allclose(row[1:4], N1 * np.array([y, z, x]), atol=1e-15)
        c = math.sqrt(15 / (4 * math.pi))
        ref2 = [c * x * y, c * y * z, math.sqrt(5 / (16 * math.pi)) * (3 * z * z - 1), c * x * z,
                math.sqrt(15 / (16 * math.pi)) * (x * x - y * y)]
        np.testing.assert_allclose(row[4:9], ref2, atol=1e-14)


def test_zlm_orthonormal_by_quadrature():
    lmax = 6
    xg, wg = np.polynomial.legendre.leggauss(16)
    nphi = 32
    G = np.zeros(((lmax + 1) ** 2,) * 2)
    for ct, w in zip(xg, wg):
        st = math.sqrt(1 - ct * ct)
        for k in range(nphi):
            ph = 2 * math.pi * k / nphi
            u = np.array([st * math.cos(ph), st * math.sin(ph), ct])
            r = O.zlm_row(lmax, u)
            G += w * (2 * math.pi / nphi) * np.outer(r, r)
    np.testing.assert_allclose(G, np.eye(len(G)), atol=1e-12)


def test_cpow_matches_integer_power():
    rng = np.random.default_rng(5)
    for _ in range(200):
        z = complex(rng.standard_normal(), rng.standard_normal())
        for n in range(7):
            assert O.cpow(z, n) == pytest.approx(z ** n, rel=1e-14, abs=1e-14)
    assert O.cpow(0j, 0) == 1 + 0j


# -- energy contract ---------------------------------------------------------------
CASES = [
    ("body2 l<=2", 2, models.biquadratic_terms(0), (2, 2, 1)),
    ("body3", 1, models.threebody_terms(0.05), (4, 1, 1)),
    ("body4", 1, models.fourbody_terms(0.05), (5, 1, 1)),
    ("chain", 1, models.chain_terms(0.05), (4, 1, 1)),
    ("mixed", 2, models.mixed_terms(7), (2, 2, 1)),
    ("high l", 1, models.highl_terms(11, 4), (3, 1, 1)),
    ("body3 l<=2", 2, models.bcc_l2_triangles(0.05e-3, np.random.default_rng(6)), (2, 2, 2)),
]


def _rand_config(n, rng):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


@pytest.mark.parametrize("name,nca,terms,dims", CASES, ids=[c[0] for c in CASES])
def test_delta_energy_is_total_energy_difference(name, nca, terms, dims):
    """test_energy.jl:19-53: exact at any body order, to round-off."""
    H = O.OracleHamiltonian(nca, terms, dims)
    rng = np.random.default_rng(3)
    cfg = _rand_config(H.n_sites, rng)
    z = H.zrows(cfg)
    E0 = H.total_energy(cfg)
    worst = 0.0
    for _ in range(6):
        s = int(rng.integers(1, H.n_sites + 1))
        e2 = _rand_config(1, rng)[0]
        c = H.site_coeffs(s, z)
        dE = H.delta_energy(c, z[s - 1], O.zlm_row(H.lmax, e2))
        cfg2 = cfg.copy()
        cfg2[s - 1] = e2
        worst = max(worst, abs(dE - (H.total_energy(cfg2) - E0)))
    assert worst < 1e-13


def test_delta_energy_keeps_accuracy_when_small():
    """test_energy.jl:68-83: the row-difference form vs an exact rational sum."""
    rng = np.random.default_rng(90210)
    n = 64
    c = rng.standard_normal(n)
    zold = 1e3 * rng.standard_normal(n)
    znew = zold + 1e-6 * rng.standard_normal(n)
    exact = sum(Fraction(c[k]) * (Fraction(znew[k]) - Fraction(zold[k])) for k in range(n))
    H = O.OracleHamiltonian(1, models.chain_terms(0.05), (4, 1, 1))
    impl = O.lib().or_delta_energy(n, O._p(c, O.C.c_double), O._p(zold, O.C.c_double), O._p(znew, O.C.c_double))
    naive = float(c @ znew - c @ zold)
    e_impl = abs(Fraction(impl) - exact)
    e_naive = abs(Fraction(naive) - exact)
    assert abs(float(exact)) > 1e-7
    assert e_impl < Fraction(1e-14) * abs(exact)
    assert e_naive > 1000 * e_impl
    del H


@pytest.mark.parametrize("name,nca,terms,dims", CASES, ids=[c[0] for c in CASES])
def test_program_kernels_equal_reference_kernels(name, nca, terms, dims):
    """test_energy.jl:143-176 (bitwise)."""
    H = O.OracleHamiltonian(nca, terms, dims)
    rng = np.random.default_rng(7)
    for _ in range(2):
        cfg = _rand_config(H.n_sites, rng)
        z = H.zrows(cfg)
        assert H.total_energy_rows(z) == H.total_energy_ref(cfg)
        for s in range(1, H.n_sites + 1):
            assert np.array_equal(H.site_coeffs(s, z), H.site_coeffs(s, z, ref=True))


def test_site_coeffs_independent_of_own_spin():
    H = O.OracleHamiltonian(2, models.biquadratic_terms(0), (2, 2, 1))
    rng = np.random.default_rng(3)
    cfg = _rand_config(H.n_sites, rng)
    for s in (1, H.n_sites):
        c1 = H.site_coeffs(s, H.zrows(cfg))
        cfg2 = cfg.copy()
        cfg2[s - 1] = _rand_config(1, rng)[0]
        assert np.array_equal(c1, H.site_coeffs(s, H.zrows(cfg2)))


def test_entry_walk_matches_site_coeffs():
    """test_gpu.jl:135-178: lane-strided direct-dE walk vs c . dZ (scaled 1e-12)."""
    rng = np.random.default_rng(31)
    for nca, terms, dims, kw in [(2, models.biquadratic_terms(3), (2, 2, 2), {}),
                                 (1, models.threebody_terms(0.05), (4, 2, 2), {}),
                                 (1, models.fourbody_terms(0.03), (4, 2, 2), {}),
                                 (4, models.dimer_terms(), (2, 1, 1),
                                  dict(magmoms=[2.2, 2.2, 1.0, 0.0], field=[0.3, -1.2, 2.0]))]:
        H = O.OracleHamiltonian(nca, terms, dims, **kw)
        cfg = _rand_config(H.n_sites, rng)
        z = H.zrows(cfg)
        for s in H.array("color_sites")[:32]:
            zn = O.zlm_row(H.lmax, _rand_config(1, rng)[0])
            c = H.site_coeffs(int(s), z)
            ref = H.delta_energy(c, z[s - 1], zn)
            scale = np.abs(c).sum() * (np.abs(zn).sum() + np.abs(z[s - 1]).sum())
            for ws in (4, 32):
                walk = sum(H.entry_walk_partial(z, zn, int(s), lane, ws) for lane in range(1, ws + 1))
                assert abs(walk - ref) <= 1e-12 * max(scale, 1e-30)


@pytest.mark.parametrize("name,nca,terms,dims", CASES[:4], ids=[c[0] for c in CASES[:4]])
def test_colouring_proper_and_partition(name, nca, terms, dims):
    H = O.OracleHamiltonian(nca, terms, dims)
    cp, cs = H.array("color_ptr"), H.array("color_sites")
    colors = np.zeros(H.n_sites, int)
    for c in range(H.n_colors):
        colors[cs[cp[c] - 1:cp[c + 1] - 1] - 1] = c + 1
    ip, isites = H.array("inst_ptr"), H.array("inst_sites")
    for i in range(len(ip) - 1):
        mem = isites[ip[i] - 1:ip[i + 1] - 1] - 1
        assert len(set(colors[mem])) == len(mem)
    assert np.array_equal(np.sort(cs), np.nonzero(H.array("site_active"))[0] + 1)
    assert cp[-1] - 1 == H.n_active


def test_keyed_sweep_drift_and_repeat_identity():
    """test_gpu.jl:253-296: repeat identity, seeds differ, drift <= 1e-8 after 200 sweeps."""
    H = O.OracleHamiltonian(2, models.biquadratic_terms(3), (2, 2, 2))
    rng = np.random.default_rng(7)
    cfg0 = _rand_config(H.n_sites, rng)
    finals = []
    for seed in (0xC0FFEE, 0xC0FFEE, 0xC0FFEF):
        cfg = cfg0.copy()
        z = H.zrows(cfg)
        E = H.total_energy(cfg)
        for sw in range(1, 201):
            _, dE, _ = H.keyed_sweep(cfg, z, 1 / 0.05, 0.6, seed, sw, 32)
            E += H.reduce_dE(dE)
        finals.append((cfg.copy(), E))
        Et = H.total_energy(cfg)
        assert abs(E - Et) <= 1e-8 * max(1.0, abs(Et))
    assert np.array_equal(finals[0][0], finals[1][0]) and finals[0][1] == finals[1][1]
    assert not np.array_equal(finals[0][0], finals[2][0])


def test_inactive_sites_frozen():
    H = O.OracleHamiltonian(4, models.dimer_terms(), (1, 1, 1))
    assert H.n_active < H.n_sites
    rng = np.random.default_rng(7)
    cfg = _rand_config(H.n_sites, rng)
    z = H.zrows(cfg)
    cfg0 = cfg.copy()
    for sw in range(1, 51):
        H.keyed_sweep(cfg, z, 20.0, 0.6, 5, sw, 4)
    assert np.array_equal(cfg[2:], cfg0[2:])


# -- closed-form statistics with the oracle's run_mc ------------------------------------
def test_dimer_energy_is_langevin():
    """<E> = J L(beta|J|) for the classical Heisenberg dimer (test_metropolis.jl:10-29)."""
    J = -0.02
    H = O.OracleHamiltonian(4, models.dimer_terms(J))
    rng = np.random.default_rng(101)
    for betaJ in (1.0, 2.5):
        ch = O.OracleChain(H, _rand_config(H.n_sites, rng), seed=100 + int(betaJ * 10), step=0.6)
        st = ch.run_mc(abs(J) / betaJ, 500, 20000, measure_interval=5)
        E, err = st["energy"][0][0], st["energy"][1][0]
        exact = J * langevin(betaJ)
        assert abs(E - exact) < 0.03 * abs(J)
        assert abs(E - exact) < 5 * max(err, 1e-3 * abs(J))
        np.testing.assert_array_equal(st["sublattice_m"][0][6:12], np.zeros(6))


def test_single_site_langevin():
    """<e_z> = -L(beta h) for h e_z (test_metropolis.jl:31-49), read off <E> = h <e_z>."""
    c0 = 0.3
    h = c0 * scemc.N1
    H = O.OracleHamiltonian(1, models.single_site_terms(c0))
    for i, bh in enumerate((1.0, 2.0)):
        ch = O.OracleChain(H, np.array([[0.0, 0.0, 1.0]]), seed=200 + i)
        st = ch.run_mc(h / bh, 500, 40000, measure_interval=2)
        assert st["energy"][0][0] / h == pytest.approx(-langevin(bh), abs=0.03)


def test_overrelaxation_pure_l1_is_microcanonical():
    """test_overrelaxation.jl:17-34: pure l = 1 reflections conserve the energy and
    are always accepted (only the two coupled dimer sites carry an l = 1 channel)."""
    H = O.OracleHamiltonian(4, models.dimer_terms())
    ch = O.OracleChain(H, _rand_config(4, np.random.default_rng(9)), seed=11)
    ch.sweeps(1 / 0.01, 5, n_or=3)
    cfg, E, _, cnt, _ = ch.get()
    assert cnt[3] == 5 * 3 * 2 and cnt[2] == cnt[3]
    assert abs(E - H.total_energy(cfg)) < 1e-12


def test_swap_rule_sign():
    """pt.jl:92-96: the colder rung holding the higher energy always swaps."""
    assert O.swap_accepts(0.1, 0.2, -1.0, -2.0, 0.999999)
    assert not O.swap_accepts(0.1, 0.2, -2.0, -1.0, 0.5)
    w = math.exp((1 / 0.1 - 1 / 0.2) * (-2.0 + 1.0))
    assert O.swap_accepts(0.1, 0.2, -2.0, -1.0, w * 0.999)
    assert not O.swap_accepts(0.1, 0.2, -2.0, -1.0, w * 1.001)


def test_adapt_step_law():
    """_adapt_step! (updates.jl:296-305): step <- clamp(step exp((a - target) / 2), 1e-3,
    pi) with a the window's Metropolis acceptance; no attempts, no change."""
    assert O.adapt_step(0.6, 50, 100, 0.5) == 0.6
    assert O.adapt_step(0.6, 100, 100, 0.5) == pytest.approx(0.6 * math.exp(0.25), rel=1e-15)
    assert O.adapt_step(0.6, 10, 100, 0.3) == pytest.approx(0.6 * math.exp(-0.1), rel=1e-15)
    assert O.adapt_step(3.1, 100, 100, 0.5) == math.pi
    assert O.adapt_step(1.1e-3, 0, 100, 0.5) == 1e-3
    assert O.adapt_step(0.6, 0, 0, 0.5) == 0.6


def test_logbinner_tau_of_ar1():
    rng = np.random.default_rng(1)
    rho, n = 0.8, 1 << 17
    x = np.zeros(n)
    e = rng.standard_normal(n)
    for i in range(1, n):
        x[i] = rho * x[i - 1] + e[i]
    m, err, tau = O.logbinner_stats(x)
    # the plateau level holds 32..63 bins, so tau carries ~30% statistical noise
    assert tau == pytest.approx(rho / (1 - rho), rel=0.5)
    assert abs(m) < 5 * err
    # the host binner of the package reproduces the oracle's cascade
    b = scemc.LogBinner(1)
    b.push_many(x[: n // 3])
    b.push_many(x[n // 3:])
    assert b.mean()[0] == pytest.approx(m, rel=1e-12, abs=1e-15)
    assert b.std_error()[0] == pytest.approx(err, rel=1e-9)
    assert b.tau_int()[0] == pytest.approx(tau, rel=1e-9)


def test_gradient_row_and_all_site_gradient_match_finite_differences():
    """The tangent gradient of every tesseral row (grad_device.jl:27-67) and the
    all-site energy gradient (gpu_gradient.jl semantics) against central finite
    differences along the two tangent directions of each spin."""
    rng = np.random.default_rng(3)
    for lmax in (1, 2, 4, 6):
        u = rng.standard_normal(3)
        u /= np.linalg.norm(u)
        g = O.grad_zlm_row(lmax, u)
        assert np.allclose(g @ u, 0.0, atol=1e-12)  # tangent
        t1 = np.cross(u, [1.0, 0.0, 0.0])
        t1 /= np.linalg.norm(t1)
        t2 = np.cross(u, t1)
        h = 1e-6
        for t in (t1, t2):
            zp = O.zlm_row(lmax, (u + h * t) / np.linalg.norm(u + h * t))
            zm = O.zlm_row(lmax, (u - h * t) / np.linalg.norm(u - h * t))
            np.testing.assert_allclose(g @ t, (zp - zm) / (2 * h), atol=2e-7, rtol=1e-6)
    from scemc import models
    OH = O.OracleHamiltonian(2, models.config2_bcc_l2().terms, (2, 2, 2), magmoms=[2.0, 2.0], field=[0, 0, 1.0])
    cfg = models.random_config(OH.n_sites, 4)
    G = OH.energy_gradient(cfg)
    h = 1e-6
    for s in (0, 5, 11):
        e = cfg[s]
        t1 = np.cross(e, [0.0, 1.0, 0.0])
        t1 /= np.linalg.norm(t1)
        for t in (t1, np.cross(e, t1)):
            cp, cm = cfg.copy(), cfg.copy()
            cp[s] = (e + h * t) / np.linalg.norm(e + h * t)
            cm[s] = (e - h * t) / np.linalg.norm(e - h * t)
            fd = (OH.total_energy(cp) - OH.total_energy(cm)) / (2 * h)
            assert G[s] @ t == pytest.approx(fd, rel=1e-5, abs=1e-10)
