"""Statistics of the device samplers against the FP64 oracle's run_mc / run_pt at the
benchmark configurations' own temperatures (run on a B200: -m gpu).

Every observable is compared through z = |mean_gpu - mean_oracle| / sqrt(err_gpu^2 +
err_oracle^2) with the log-binning / jackknife error bars of both sides. The contract is
agreement within 2 sigma per observable; with many observables some z exceed 2 by chance
(about 5 % of them when the error bars are right), so the gate is the statement that the
z-scores are those of agreeing samplers: at most 10 % of them above 2, none above 3.5, and
sum z^2 below the 99th percentile of chi^2 with one degree of freedom per comparison.

Both models have anisotropic couplings (random l <= 2 pair tensors, odd-order l = 1
triangles), so their ordered phases have a preferred magnetisation direction and, from a
random start, low-temperature chains settle into different long-lived orientations. Both
samplers therefore start from the same state, ordered along the direction whose uniform
state has the lowest energy (learned.easy_axis), and are compared at equilibrium.
"""
import numpy as np
import pytest
from scipy import stats as sps

import oracle as O
import scemc
from scemc import learned, models

pytestmark = pytest.mark.gpu


def zscores(a, b, names, comps=None):
    out = []
    for n in names:
        ma = np.atleast_1d(np.asarray(a[n].mean, float))
        ea = np.atleast_1d(np.asarray(a[n].err, float))
        mb, eb = np.atleast_1d(np.asarray(b[n][0], float)), np.atleast_1d(np.asarray(b[n][1], float))
        if comps and n in comps:
            ma, ea, mb, eb = ma[comps[n]], ea[comps[n]], mb[comps[n]], eb[comps[n]]
        out += list(np.abs(ma - mb) / np.sqrt(ea ** 2 + eb ** 2 + 1e-300))
    return out


def assert_consistent(zs, label):
    zs = np.asarray(zs, float)
    chi2 = float(np.sum(zs ** 2))
    p = float(sps.chi2.sf(chi2, len(zs)))
    over = float(np.mean(zs > 2.0))
    msg = f"{label}: chi2 {chi2:.1f} over {len(zs)}, p {p:.3g}; z = " + " ".join(f"{z:.2f}" for z in zs)
    assert zs.max() < 3.5 and over <= 0.10 and p > 0.01, msg


def test_config2_statistics_at_its_temperatures(gpu):
    """The second configuration's model (bcc, l <= 2 pairs to shell 3, l = 1 plaquettes,
    Zeeman 2 muB in 1 T along z) on a 4^3 lattice at its five temperatures, kT uniform in
    [0.2, 2.0] meV, Metropolis + 1 overrelaxation pass per sweep: energy, |m| and the
    field-aligned sublattice magnetisations of the device chains against the oracle's
    run_mc at each temperature."""
    w = models.config2_bcc_l2(n=4)
    H = w.hamiltonians()[0]
    OH = O.OracleHamiltonian(2, w.terms, (4, 4, 4), magmoms=w.magmoms, field=w.field)
    gH = scemc.GPUTiledHamiltonian(H)
    n_star = learned.easy_axis(gH)
    start = np.tile(n_star, (H.n_sites, 1))
    r = scemc.gpu_run_pt(gH, kT=w.kts, exchange=False, sweeps_therm=4000, sweeps_measure=20000,
                         or_per_metropolis=1, seed=21, init=n_star)
    zs = []
    for i, (kT, p) in enumerate(zip(w.kts, r.points)):
        ost = O.OracleChain(OH, start, seed=210 + i).run_mc(float(kT), 4000, 20000, n_or=1)
        zs += zscores(p.stats, ost, ["energy", "absm", "sublattice_m"], comps={"sublattice_m": [2, 5]})
        assert abs(p.acceptance_or - ost["acceptance_or"]) < 0.02, (float(kT), p.acceptance_or, ost["acceptance_or"])
    assert len(zs) == 20
    assert_consistent(zs, "config 2")


def test_config3_ladders_on_8_and_12_cubed(gpu):
    """The batched parallel-tempering configuration's ladder (16 rungs, kT geometric in
    [0.1, 3.0] meV, J1/J2 isotropic l = 1 plus (NN, NN, NNN) triangles, swaps after every
    sweep) on its 8^3 and 12^3 chains, both ladders in one device batch: energy and |m| of
    every rung against the oracle's run_pt of each ladder, and the swap acceptance of every
    rung pair."""
    w = models.config3_bcc_pt()
    Hs = [scemc.TiledHamiltonian(2, w.terms, dims=(n, n, n)) for n in (8, 12)]
    gHs = [scemc.GPUTiledHamiltonian(H) for H in Hs]
    n_star = learned.easy_axis(scemc.GPUTiledHamiltonian(scemc.TiledHamiltonian(2, w.terms, dims=(4, 4, 4))))
    r = scemc.gpu_run_pt(gHs, kT=w.kts, exchange_interval=1, sweeps_therm=2000, sweeps_measure=10000, seed=31,
                         init=n_star)
    threads = max(1, min(16, O.lib().or_max_threads()))
    zs = []
    for li, (n, H) in enumerate(zip((8, 12), Hs)):
        OH = O.OracleHamiltonian(2, w.terms, (n, n, n))
        start = np.tile(n_star, (H.n_sites, 1))
        chains = [O.OracleChain(OH, start, seed=3100 + 16 * li + i) for i in range(len(w.kts))]
        pts, swaps = O.run_pt(OH, chains, w.kts, 2000, 10000, exchange_interval=1, threads=threads)
        for p, q in zip(r.points[16 * li:16 * (li + 1)], pts):
            zs += zscores(p.stats, q, ["energy", "absm"])
        gpu_swaps = r.swap_acceptance[15 * li:15 * (li + 1)]
        np.testing.assert_allclose(gpu_swaps, swaps, atol=0.05)
    assert len(zs) == 64
    assert_consistent(zs, "config 3 ladders")
