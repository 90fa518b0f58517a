"""Synthetic SCE term lists: the five benchmark workloads and the reference's
hand-built test fixtures.

No fitted model can be loaded here (SCEFitting is not available), so every model is
a seeded `MultipoleTerm` list with the shapes of the workloads it stands for.
Couplings are given in meV and converted to eV (the reference's units, with
`KB_EV` / `MU_B_EV_T`). An isotropic l = 1 pair with `folded = I3` and raw
coefficient c has energy 3c (e_i . e_j) after the (4 pi)^(body/2) scale, so a
Heisenberg bond J e_i . e_j uses c = J / 3.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass

import numpy as np

from .hamiltonian import FOUR_PI, N1, MultipoleTerm, TiledHamiltonian

MEV = 1e-3  # eV per meV

Z3 = (0, 0, 0)


# ---------------------------------------------------------------------------
# reference test fixtures (test/unit/fixtures.jl, test/unit/test_energy.jl)
# ---------------------------------------------------------------------------
def chain_terms(J: float):
    """Both directed members of the +x bond of a 1-atom chain (test/unit/fixtures.jl:94-103)."""
    folded = np.eye(3)
    raw = J / (2 * N1 ** 2 * FOUR_PI)
    return [MultipoleTerm(raw, [1, 1], [Z3, (1, 0, 0)], [1, 1], folded.copy()),
            MultipoleTerm(raw, [1, 1], [Z3, (-1, 0, 0)], [1, 1], folded.copy())]


def threebody_terms(J: float):
    """3-body chain cluster (0, +x, +2x) (test/unit/fixtures.jl:109-117); triplet fast path."""
    f = np.zeros((3, 3, 3))
    f[1, 1, 1] = 1.0
    f[0, 2, 0] = 0.7
    f[2, 0, 1] = -0.4
    return [MultipoleTerm(J, [1, 1, 1], [Z3, (1, 0, 0), (2, 0, 0)], [1, 1, 1], f)]


def fourbody_terms(J: float):
    """4-body chain cluster (0, +x, +2x, +3x) (test/unit/fixtures.jl:122-131); general path."""
    f = np.zeros((3, 3, 3, 3))
    f[1, 1, 1, 1] = 1.0
    f[0, 2, 1, 0] = 0.6
    f[2, 1, 0, 2] = -0.3
    return [MultipoleTerm(J, [1, 1, 1, 1], [Z3, (1, 0, 0), (2, 0, 0), (3, 0, 0)], [1, 1, 1, 1], f)]


def dimer_terms(J: float = -0.02):
    """Isotropic l = 1 pair between atoms 1 and 2 of a 4-atom cell; atoms 3 and 4 are
    untouched (inactive). Energy J e1 . e2 per cell (the fitted dimer of
    test/unit/fixtures.jl:27-31, restated as a hand-built term)."""
    return [MultipoleTerm(J / 3.0, [1, 2], [Z3, Z3], [1, 1], np.eye(3))]


def dimer(dims=(1, 1, 1), J: float = -0.02, **kw) -> TiledHamiltonian:
    return TiledHamiltonian(4, dimer_terms(J), dims=dims, **kw)


def biquadratic_terms(seed: int, scale: float = 0.05):
    """Anisotropic l <= 2 pair between the two atoms of a 2-atom cell: one template
    per (l1, l2) in {1,2}^2 with N(0, scale) entries (test/unit/fixtures.jl:55-61 restated)."""
    rng = np.random.default_rng(seed)
    out = []
    for l1, l2 in itertools.product((1, 2), (1, 2)):
        f = scale * rng.standard_normal((2 * l1 + 1, 2 * l2 + 1))
        out.append(MultipoleTerm(1.0 / FOUR_PI, [1, 2], [Z3, Z3], [l1, l2], f))
    return out


def mixed_terms(seed: int = 7):
    """Bodies 1+2+3 with half-sparse random tensors (test_energy.jl:150-160 shape)."""
    rng = np.random.default_rng(seed)

    def sparse(*dims):
        f = rng.standard_normal(dims)
        f[rng.random(dims) < 0.5] = 0.0
        return f

    x = (1, 0, 0)
    return [MultipoleTerm(0.3, [1], [Z3], [2], sparse(5)),
            MultipoleTerm(-0.2, [1, 2], [Z3, Z3], [1, 1], sparse(3, 3)),
            MultipoleTerm(0.1, [1, 2, 1], [Z3, Z3, x], [1, 1, 2], sparse(3, 3, 5))]


def single_site_terms(c0: float = 0.3):
    """One spin in a uniaxial l = 1 potential h e_z with h = c0 N1 (test_metropolis.jl:31-49)."""
    folded = np.zeros(3)
    folded[1] = 1.0
    return [MultipoleTerm(c0 / math.sqrt(FOUR_PI), [1], [Z3], [1], folded)]


def highl_terms(seed: int = 11, lmax: int = 4):
    """A pair chain with l up to `lmax` (exercises the general tesseral rows)."""
    rng = np.random.default_rng(seed)
    out = []
    for l1, l2 in [(1, lmax), (lmax, 2), (3, 3)]:
        f = 0.02 * rng.standard_normal((2 * l1 + 1, 2 * l2 + 1))
        out.append(MultipoleTerm(1.0 / FOUR_PI, [1, 1], [Z3, (1, 0, 0)], [l1, l2], f))
    return out


# ---------------------------------------------------------------------------
# lattice helpers
# ---------------------------------------------------------------------------
@dataclass
class Lattice:
    """A cubic conventional cell with fractional atom positions."""

    positions: np.ndarray  # (n_atoms, 3)

    @property
    def n_atoms(self) -> int:
        return len(self.positions)

    def locate(self, p):
        """(atom 1-based, integer cell) of a fractional position."""
        for a, q in enumerate(self.positions):
            d = np.asarray(p) - q
            r = np.round(d)
            if np.all(np.abs(d - r) < 1e-9):
                return a + 1, tuple(int(x) for x in r)
        raise ValueError(f"no atom at {p}")

    def neighbours(self, a: int, dist: float):
        """Vectors from atom a (1-based) to every site at distance `dist`."""
        out = []
        pa = self.positions[a - 1]
        for off in itertools.product(range(-2, 3), repeat=3):
            for q in self.positions:
                v = q + np.asarray(off) - pa
                if abs(np.linalg.norm(v) - dist) < 1e-9:
                    out.append(v)
        return out

    def shells(self, n: int):
        ds = set()
        for a in range(1, self.n_atoms + 1):
            pa = self.positions[a - 1]
            for off in itertools.product(range(-2, 3), repeat=3):
                for q in self.positions:
                    d = np.linalg.norm(q + np.asarray(off) - pa)
                    if d > 1e-9:
                        ds.add(round(d, 9))
        return sorted(ds)[:n]

    def bonds(self, dist: float):
        """Undirected bonds at `dist`, one template per bond per cell: (a, b, shift)."""
        out = []
        for a in range(1, self.n_atoms + 1):
            for v in self.neighbours(a, dist):
                if not _positive(v):
                    continue
                b, cell = self.locate(self.positions[a - 1] + v)
                out.append((a, b, cell))
        return out

    def clusters(self, members_list):
        """Deduplicate clusters given as lists of absolute fractional positions; return
        (atoms, shifts) anchored so that the first member is in the home cell."""
        seen = set()
        out = []
        for pos in members_list:
            locs = [self.locate(p) for p in pos]
            key0 = sorted(locs, key=lambda t: (t[1], t[0]))
            base = key0[0][1]
            key = tuple(sorted((a, tuple(c - b for c, b in zip(cell, base))) for a, cell in locs))
            if key in seen:
                continue
            seen.add(key)
            first = locs[0][1]
            atoms = [a for a, _ in locs]
            shifts = [tuple(c - f for c, f in zip(cell, first)) for _, cell in locs]
            out.append((atoms, shifts))
        return out


def _positive(v) -> bool:
    for x in np.round(v, 9):
        if x > 0:
            return True
        if x < 0:
            return False
    return False


SC = Lattice(np.zeros((1, 3)))
BCC = Lattice(np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]]))
FCC = Lattice(np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]))


def heisenberg_pairs(lat: Lattice, shell_J):
    """Isotropic l = 1 bonds, J (eV) per shell: E = sum J e_i . e_j."""
    dists = lat.shells(len(shell_J))
    terms = []
    for dist, J in zip(dists, shell_J):
        for a, b, cell in lat.bonds(dist):
            terms.append(MultipoleTerm(J / 3.0, [a, b], [Z3, cell], [1, 1], np.eye(3)))
    return terms


def multipole_pairs(lat: Lattice, shell_mean, sigma: float, rng, ls=(1, 2)):
    """Pairs with every (l1, l2) block, l in `ls`: isotropic l = 1 diagonal with the
    shell mean J/3, plus N(0, sigma/3) on every (l1 m1, l2 m2) entry (eV)."""
    dists = lat.shells(len(shell_mean))
    terms = []
    for dist, J in zip(dists, shell_mean):
        for a, b, cell in lat.bonds(dist):
            for l1, l2 in itertools.product(ls, ls):
                f = (sigma / 3.0) * rng.standard_normal((2 * l1 + 1, 2 * l2 + 1))
                if l1 == 1 and l2 == 1:
                    f += (J / 3.0) * np.eye(3)
                terms.append(MultipoleTerm(1.0, [a, b], [Z3, cell], [l1, l2], f))
    return terms


def bcc_triangles(sigma: float, rng):
    """bcc (NN, NN, NNN) triangles, l = 1, N(0, sigma) dense tensors (eV)."""
    nn, nnn = BCC.shells(2)
    mem = []
    for a in (1, 2):
        pa = BCC.positions[a - 1]
        for v1 in BCC.neighbours(a, nnn):
            for v2 in BCC.neighbours(a, nn):
                if abs(np.linalg.norm(v1 - v2) - nn) < 1e-9:
                    mem.append([pa, pa + v2, pa + v1])
    out = []
    for atoms, shifts in BCC.clusters(mem):
        f = sigma * rng.standard_normal((3, 3, 3)) / FOUR_PI ** 1.5
        out.append(MultipoleTerm(1.0, atoms, shifts, [1, 1, 1], f))
    return out


def bcc_l2_triangles(sigma: float, rng):
    """bcc (NN, NN, NNN) triangles with every member l in {1, 2}: one template per
    (l1, l2, l3) combination, N(0, sigma) dense tensors (eV). The reference's fitted
    models are dominated by body-3 terms of this kind (l up to 2 on every member)."""
    nn, nnn = BCC.shells(2)
    mem = []
    for a in (1, 2):
        pa = BCC.positions[a - 1]
        for v1 in BCC.neighbours(a, nnn):
            for v2 in BCC.neighbours(a, nn):
                if abs(np.linalg.norm(v1 - v2) - nn) < 1e-9:
                    mem.append([pa, pa + v2, pa + v1])
    out = []
    for atoms, shifts in BCC.clusters(mem):
        for ls in itertools.product((1, 2), repeat=3):
            f = sigma * rng.standard_normal(tuple(2 * l + 1 for l in ls)) / FOUR_PI ** 1.5
            out.append(MultipoleTerm(1.0, atoms, shifts, list(ls), f))
    return out


def sc_plaquettes(lat: Lattice, sigma: float, rng):
    """4-site squares of each atom's simple-cubic sublattice (three planes per atom),
    l = 1, N(0, sigma) dense tensors (eV)."""
    out = []
    e = np.eye(3, dtype=int)
    for a in range(1, lat.n_atoms + 1):
        for i, j in ((0, 1), (1, 2), (2, 0)):
            shifts = [Z3, tuple(e[i]), tuple(e[i] + e[j]), tuple(e[j])]
            f = sigma * rng.standard_normal((3, 3, 3, 3)) / FOUR_PI ** 2
            out.append(MultipoleTerm(1.0, [a] * 4, shifts, [1, 1, 1, 1], f))
    return out


def fcc_nn_triangles(sigma: float, rng):
    nn = FCC.shells(1)[0]
    mem = []
    for a in range(1, 5):
        pa = FCC.positions[a - 1]
        vs = FCC.neighbours(a, nn)
        for v1, v2 in itertools.combinations(vs, 2):
            if abs(np.linalg.norm(v1 - v2) - nn) < 1e-9:
                mem.append([pa, pa + v1, pa + v2])
    out = []
    for atoms, shifts in FCC.clusters(mem):
        f = sigma * rng.standard_normal((3, 3, 3)) / FOUR_PI ** 1.5
        out.append(MultipoleTerm(1.0, atoms, shifts, [1, 1, 1], f))
    return out


# ---------------------------------------------------------------------------
# the five benchmark workloads
# ---------------------------------------------------------------------------
@dataclass
class Workload:
    name: str
    n_cell_atoms: int
    terms: list
    dims_list: list          # one supercell per ladder / chain family
    kts: np.ndarray          # temperatures (eV) per replica of one ladder
    magmoms: object = None
    field: object = None
    sweeps_therm: int = 0
    sweeps_measure: int = 0
    or_per_metropolis: int = 0
    seed: int = 0
    exchange: bool = False

    def hamiltonians(self):
        return [TiledHamiltonian(self.n_cell_atoms, self.terms, dims=d, magmoms=self.magmoms, field=self.field)
                for d in self.dims_list]


def config1_sc(n: int = 8) -> Workload:
    """sc n^3, J1 = -1.0 meV (NN), J2 = -0.2 meV (NNN), kT = 0.5 meV, seed 1."""
    terms = heisenberg_pairs(SC, [-1.0 * MEV, -0.2 * MEV])
    return Workload("sc8_J1J2", 1, terms, [(n, n, n)], np.array([0.5 * MEV]), sweeps_therm=2000,
                    sweeps_measure=20000, seed=1)


def config2_bcc_l2(n: int = 16) -> Workload:
    """bcc 2-sublattice n^3: l<=2 pairs to shell 3 (means -1.0/-0.3/-0.1 meV, sigma 0.1 meV),
    l=1 plaquettes N(0, 0.05 meV), Zeeman 2 muB in 1 T || z; 5 kT in [0.2, 2.0] meV; seed 2."""
    rng = np.random.default_rng(2)
    terms = multipole_pairs(BCC, [-1.0 * MEV, -0.3 * MEV, -0.1 * MEV], 0.1 * MEV, rng)
    terms += sc_plaquettes(BCC, 0.05 * MEV, rng)
    kts = np.linspace(0.2, 2.0, 5) * MEV
    return Workload("bcc16_l2_plaq_zeeman", 2, terms, [(n, n, n)], kts, magmoms=[2.0, 2.0],
                    field=[0.0, 0.0, 1.0], sweeps_therm=2000, sweeps_measure=10000, or_per_metropolis=1, seed=2)


def config3_bcc_pt(sizes=(8, 12, 16, 24), rungs: int = 16) -> Workload:
    """4 PT ladders (one per bcc size) of `rungs` rungs, kT geometric in [0.1, 3.0] meV:
    J1/J2 isotropic l=1 + (NN,NN,NNN) triangles N(0, 0.1 meV); swaps every sweep; seed 3."""
    rng = np.random.default_rng(3)
    terms = heisenberg_pairs(BCC, [-1.0 * MEV, -0.2 * MEV]) + bcc_triangles(0.1 * MEV, rng)
    kts = np.geomspace(0.1, 3.0, rungs) * MEV
    return Workload("bcc_pt_uneven", 2, terms, [(s, s, s) for s in sizes], kts, sweeps_therm=2000,
                    sweeps_measure=8000, seed=3, exchange=True)


def bcc_l2_body3(n: int = 16) -> Workload:
    """bcc n^3 with l <= 2 pairs to shell 2 (means -1.0/-0.3 meV, sigma 0.1 meV) and
    (NN, NN, NNN) triangles with every (l1, l2, l3) in {1, 2}^3, N(0, 0.05 meV); 5 kT in
    [0.2, 2.0] meV; Metropolis + OR; seed 6. The body-3-with-l = 2 regime of fitted
    models (not one of the five benchmark configurations)."""
    rng = np.random.default_rng(6)
    terms = multipole_pairs(BCC, [-1.0 * MEV, -0.3 * MEV], 0.1 * MEV, rng)
    terms += bcc_l2_triangles(0.05 * MEV, rng)
    kts = np.linspace(0.2, 2.0, 5) * MEV
    return Workload("bcc16_l2_body3", 2, terms, [(n, n, n)], kts, sweeps_therm=2000, sweeps_measure=10000,
                    or_per_metropolis=1, seed=6)


def config4_bcc_body4(n: int = 32) -> Workload:
    """bcc n^3: J1/J2 isotropic l=1 + l=1 plaquettes N(0, 0.05 meV); seed 4."""
    rng = np.random.default_rng(4)
    terms = heisenberg_pairs(BCC, [-1.0 * MEV, -0.2 * MEV]) + sc_plaquettes(BCC, 0.05 * MEV, rng)
    kts = np.geomspace(0.2, 2.0, 16) * MEV
    return Workload("bcc32_body4", 2, terms, [(n, n, n)], kts, sweeps_therm=2000, sweeps_measure=10000, seed=4)


def config5_fcc(n: int = 64, replicas: int = 32) -> Workload:
    """fcc 4-site cell n^3: l<=2 pairs to shell 4, N(0, 1.0 meV) with +0.5 meV shell-1
    isotropic mean; NN triangles N(0, 0.1 meV); Zeeman 2 muB, 0.5 T || [111];
    `replicas` PT rungs, kT in [0.05, 2.0] meV; OR; seed 5."""
    rng = np.random.default_rng(5)
    terms = multipole_pairs(FCC, [0.5 * MEV, 0.0, 0.0, 0.0], 1.0 * MEV, rng)
    terms += fcc_nn_triangles(0.1 * MEV, rng)
    b = 0.5 / math.sqrt(3.0)
    kts = np.geomspace(0.05, 2.0, replicas) * MEV
    return Workload("fcc64_l2_tri_zeeman", 4, terms, [(n, n, n)], kts, magmoms=[2.0] * 4, field=[b, b, b],
                    sweeps_therm=1000, sweeps_measure=4000, or_per_metropolis=1, seed=5, exchange=True)


def random_config(n_sites: int, seed: int) -> np.ndarray:
    """Uniform random unit spins, 3 x n column-major (n x 3 row-major array)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n_sites, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)
