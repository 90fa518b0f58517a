"""Learned proposal: the per-site network, its training data and the environment
table (no counterpart in the reference; the acceptance it feeds is the
reference's Metropolis test of src/updates.jl:37-64 with the Hastings factor
q(e | env) / q(e' | env), so the stationary distribution is unchanged).

The network (3 n_env + 1 -> 128 -> 128 -> 20, SiLU; 43 inputs for the 14-site
bcc environment, 55 for the 18-site fcc one) and its training run in
libscemc_cuda.so on the tcgen05 tensor cores; this module is the host side.
"""
from __future__ import annotations

import ctypes as C
import itertools

import numpy as np

from . import _lib
from ._lib import F32P, F64P, check, ptr

N_PARAMS = 28960
N_IN, N_OUT = 43, 20
MEV = 1e-3

# (name, offset, shape) of the parameter block
LAYOUT = [("W1", 0, (128, 64)), ("b1", 8192, (128,)), ("W2", 8320, (128, 128)), ("b2", 24704, (128,)),
          ("W3", 24832, (32, 128)), ("b3", 28928, (32,))]


def unpack(flat: np.ndarray) -> dict:
    return {n: flat[o:o + int(np.prod(s))].reshape(s) for n, o, s in LAYOUT}


def pack(P: dict) -> np.ndarray:
    flat = np.zeros(N_PARAMS, np.float32)
    for n, o, s in LAYOUT:
        flat[o:o + int(np.prod(s))] = np.asarray(P[n], np.float32).reshape(-1)
    return flat


class ProposalNet:
    """The learned proposal network (device resident). Environment mode: n_in = 3 n_env
    + 1 inputs (n_env environment spins, then kT in meV). Field mode (field_rows = 3 for
    lmax 1, 8 for lmax 2): n_in = field_rows + 1 inputs, the site's leave-one-out
    coefficients in meV and kT in meV; they fix the site's conditional distribution
    whatever the range of the couplings."""

    def __init__(self, seed: int = 0, n_env: int = 14, field_rows: int = 0):
        if field_rows:
            if field_rows not in (3, 8):
                raise ValueError("field_rows must be 3 (lmax 1) or 8 (lmax 2)")
            self.n_env = 0
            self.n_in = int(field_rows) + 1
        else:
            if not 1 <= n_env <= 21:
                raise ValueError("n_env must be 1..21")
            self.n_env = int(n_env)
            self.n_in = 3 * self.n_env + 1
        h = C.c_void_p()
        check(_lib.lib().scemc_mlp_create(int(seed) & (2 ** 64 - 1), self.n_in, C.byref(h)))
        self.h = h

    def _rows(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        if X.ndim != 2 or X.shape[1] != self.n_in:
            raise ValueError(f"inputs must be (n, {self.n_in})")
        return X

    def __del__(self):
        if getattr(self, "h", None):
            try:
                _lib.lib().scemc_mlp_destroy(self.h)
            except Exception:  # interpreter shutdown: the module may already be gone
                pass
            self.h = None

    def params(self) -> np.ndarray:
        out = np.zeros(N_PARAMS, np.float32)
        check(_lib.lib().scemc_mlp_get_params(self.h, ptr(out, C.c_float)))
        return out

    def set_params(self, flat) -> None:
        flat = np.ascontiguousarray(flat, np.float32)
        if flat.size != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters")
        check(_lib.lib().scemc_mlp_set_params(self.h, ptr(flat, C.c_float)))

    def forward(self, X) -> np.ndarray:
        X = self._rows(X)
        n = X.shape[0]
        out = np.zeros((n, N_OUT), np.float32)
        check(_lib.lib().scemc_mlp_forward(self.h, ptr(X, C.c_float), n, ptr(out, C.c_float)))
        return out

    def loss_grad(self, X, Y):
        X = self._rows(X)
        Y = np.ascontiguousarray(Y, np.float32)
        loss = C.c_double()
        g = np.zeros(N_PARAMS, np.float32)
        check(_lib.lib().scemc_mlp_loss_grad(self.h, ptr(X, C.c_float), ptr(Y, C.c_float), X.shape[0],
                                             C.byref(loss), ptr(g, C.c_float)))
        return loss.value, g

    def train(self, X, Y, batch: int = 1024, epochs: int = 10, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        """Adam on shuffled minibatches; returns each epoch's mean minibatch loss."""
        X = self._rows(X)
        Y = np.ascontiguousarray(Y, np.float32)
        losses = np.zeros(max(epochs, 1))
        check(_lib.lib().scemc_mlp_train(self.h, ptr(X, C.c_float), ptr(Y, C.c_float), X.shape[0], int(batch),
                                         int(epochs), float(lr), int(seed) & (2 ** 64 - 1), ptr(losses, C.c_double)))
        return losses[:epochs]


def environment_table(positions: np.ndarray, dims, n_shells: int = 2, tol: float = 1e-6) -> np.ndarray:
    """Canonical environment of every site: the sites of the first `n_shells`
    neighbour shells, ordered by displacement vector (lexicographic in x, y, z).
    positions: fractional atom positions of the cubic cell (n_atoms, 3); site
    numbering as TiledHamiltonian.site_index (0-based here). Returns (n_sites, K)
    int32."""
    pos = np.asarray(positions, float)
    na = pos.shape[0]
    d1, d2, d3 = (int(x) for x in dims)
    # displacement list per atom: all (atom b, cell offset) within the shell radii
    cands = []
    for a in range(na):
        lst = []
        for off in itertools.product(range(-2, 3), repeat=3):
            for b in range(na):
                v = pos[b] + np.asarray(off) - pos[a]
                r = float(np.linalg.norm(v))
                if r > tol:
                    lst.append((r, tuple(np.round(v, 9)), b, off))
        cands.append(lst)
    radii = sorted({round(c[0], 6) for c in cands[0]})[:n_shells]
    rmax = radii[-1] + tol
    per_atom = []
    for a in range(na):
        sel = sorted([c for c in cands[a] if c[0] <= rmax], key=lambda c: c[1])
        per_atom.append(sel)
    K = len(per_atom[0])
    if any(len(p) != K for p in per_atom):
        raise ValueError("sublattices have different environment sizes")
    n_sites = na * d1 * d2 * d3
    env = np.zeros((n_sites, K), np.int32)
    for c2 in range(d3):
        for c1 in range(d2):
            for c0 in range(d1):
                for a in range(na):
                    s = a + na * (c0 + d1 * (c1 + d2 * c2))
                    for k, (_, _, b, off) in enumerate(per_atom[a]):
                        t0 = (c0 + off[0]) % d1
                        t1 = (c1 + off[1]) % d2
                        t2 = (c2 + off[2]) % d3
                        env[s, k] = b + na * (t0 + d1 * (t1 + d2 * t2))
    return env


def environment_rows(configs, env: np.ndarray, kts_ev, sites=None) -> np.ndarray:
    """Network inputs (n, 3 k + 1) for the given sites of each configuration: the
    k environment spins in table order, then kT in meV."""
    rows = []
    for cfg, kt in zip(configs, kts_ev):
        cfg = np.asarray(cfg).reshape(-1, 3)
        ss = np.arange(cfg.shape[0]) if sites is None else np.asarray(sites)
        x = cfg[env[ss]].reshape(len(ss), -1)
        rows.append(np.concatenate([x, np.full((len(ss), 1), kt / MEV)], axis=1))
    return np.concatenate(rows).astype(np.float32)


def collect_training_set(H, env, kts, n_rows: int, *, sweeps_therm: int = 2000, snapshots: int = 4,
                         spacing: int = 50, seed: int = 0, kernel: int = 0, init=None):
    """Site environments from plain-Metropolis chains, one per kT (one batch on the
    device): after `sweeps_therm` adaptive-step sweeps from random spins (or from
    `init`, one configuration for every chain), `snapshots` configurations `spacing`
    sweeps apart; n_rows rows drawn evenly over kT values and snapshots.
    Returns (X (n, 3 k + 1) float32, Y (n, 3) float32): inputs and the site's own spin."""
    from .gpu import GPUBatch, GPUTiledHamiltonian
    gH = H if isinstance(H, GPUTiledHamiltonian) else GPUTiledHamiltonian(H)
    host = gH.host
    rng = np.random.default_rng(seed)
    R = len(kts)
    cfgs = []
    for _ in range(R):
        if init is not None:
            cfgs.append(np.asarray(init, np.float64).reshape(-1, 3).copy())
            continue
        v = rng.standard_normal((host.n_sites, 3))
        cfgs.append(v / np.linalg.norm(v, axis=1, keepdims=True))
    b = GPUBatch([gH], [R], cfgs, rng.integers(0, 2 ** 63, size=R).tolist(), 0.6)
    b.set_betas(1.0 / np.asarray(kts))
    b.run(sweeps_therm, adapt_interval=50, adapt_target=0.5, phase_total=sweeps_therm, kernel=kernel)
    per = int(np.ceil(n_rows / (R * snapshots)))
    X, Y = [], []
    for _ in range(snapshots):
        b.run(spacing, kernel=kernel)
        st = b.download()
        for r in range(R):
            cfg = st["configs"][st["slot_of_rung"][r]]
            sites = rng.choice(host.n_sites, size=per, replace=per > host.n_sites)
            X.append(environment_rows([cfg], env, [kts[r]], sites))
            Y.append(np.asarray(cfg)[sites].astype(np.float32))
    X = np.concatenate(X)[:n_rows]
    Y = np.concatenate(Y)[:n_rows]
    return X, Y


def fibonacci_sphere(n: int) -> np.ndarray:
    """n nearly uniform unit vectors (golden-angle spiral), (n, 3)."""
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    ph = np.pi * (3.0 - np.sqrt(5.0)) * i
    return np.stack([r * np.cos(ph), r * np.sin(ph), z], axis=1)


def ordered_energies(gH, directions) -> np.ndarray:
    """FP64 energy per site of the uniform states e_s = n for each direction n (one
    device batch, one replica per direction; the library's energy recompute)."""
    from .gpu import GPUBatch
    d = np.asarray(directions, np.float64).reshape(-1, 3)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    ns = gH.n_sites
    out = []
    for i in range(0, len(d), 512):  # a batch holds at most 512 replica slots
        part = d[i:i + 512]
        cfgs = [np.broadcast_to(v, (ns, 3)) for v in part]
        b = GPUBatch([gH], [len(part)], cfgs, np.arange(1, len(part) + 1), 0.6)
        out.append(b.download()["energies"] / gH.host.n_active)
    return np.concatenate(out)


def easy_axis(gH, n_dirs: int = 4096, rounds: int = 3) -> np.ndarray:
    """The direction n that minimises the energy of the uniform state e_s = n: the
    orientation a ferromagnetically ordered chain relaxes to when anisotropic terms
    (l = 1 body-3/body-4 products with random coefficients) pick an easy axis. A
    chain started ordered along another axis has to rotate its whole magnetisation,
    which local moves do slowly on large lattices; starting along n removes that
    transient. Grid search on a Fibonacci sphere, then `rounds` refinements on
    shrinking caps around the best direction. gH should be a small lattice of the
    same model (the uniform state's energy per site does not depend on its size)."""
    dirs = fibonacci_sphere(n_dirs)
    e = ordered_energies(gH, dirs)
    best = dirs[int(np.argmin(e))]
    width = 2.0 / np.sqrt(n_dirs)
    for _ in range(rounds):
        t1 = np.cross(best, [1.0, 0.0, 0.0] if abs(best[0]) < 0.9 else [0.0, 1.0, 0.0])
        t1 /= np.linalg.norm(t1)
        t2 = np.cross(best, t1)
        g = np.linspace(-width, width, 21)
        a, c = np.meshgrid(g, g)
        cand = best + a.reshape(-1, 1) * t1 + c.reshape(-1, 1) * t2
        cand /= np.linalg.norm(cand, axis=1, keepdims=True)
        e = ordered_energies(gH, cand)
        best = cand[int(np.argmin(e))]
        width /= 8.0
    return best


def collect_field_training_set(H, kts, n_rows: int, *, sweeps_therm: int = 2000, snapshots: int = 4,
                               spacing: int = 50, seed: int = 0, kernel: int = 0, init=None,
                               or_per_metropolis: int = 0):
    """Field-mode training rows from plain-Metropolis chains, one per kT (one device
    batch): after `sweeps_therm` adaptive-step sweeps, `snapshots` configurations
    `spacing` sweeps apart; each row is a site's leave-one-out coefficients in meV
    (scemc_batch_site_coeffs) and kT in meV, its target the site's spin.
    Returns (X (n, NR + 1) float32, Y (n, 3) float32)."""
    from .gpu import GPUBatch, GPUTiledHamiltonian
    gH = H if isinstance(H, GPUTiledHamiltonian) else GPUTiledHamiltonian(H)
    host = gH.host
    rng = np.random.default_rng(seed)
    R = len(kts)
    if init is None:
        cfgs = []
        for _ in range(R):
            v = rng.standard_normal((host.n_sites, 3))
            cfgs.append(v / np.linalg.norm(v, axis=1, keepdims=True))
    else:
        c0 = np.asarray(init, np.float64).reshape(-1, 3)
        if c0.shape[0] == 1:
            c0 = np.tile(c0 / np.linalg.norm(c0), (host.n_sites, 1))
        cfgs = [c0.copy() for _ in range(R)]
    b = GPUBatch([gH], [R], cfgs, rng.integers(0, 2 ** 63, size=R).tolist(), 0.6)
    b.set_betas(1.0 / np.asarray(kts))
    b.run(sweeps_therm, adapt_interval=50, adapt_target=0.5, phase_total=sweeps_therm, kernel=kernel,
          or_per_metropolis=or_per_metropolis)
    per = int(np.ceil(n_rows / (R * snapshots)))
    X, Y = [], []
    for _ in range(snapshots):
        b.run(spacing, kernel=kernel, or_per_metropolis=or_per_metropolis)
        st = b.download()
        for r in range(R):
            slot = st["slot_of_rung"][r]
            c = b.site_coeffs(slot)
            cfg = np.asarray(st["configs"][slot])
            sites = rng.choice(host.n_sites, size=per, replace=per > host.n_sites)
            x = np.empty((per, c.shape[1] + 1), np.float32)
            x[:, :-1] = 1.0e3 * c[sites]
            x[:, -1] = kts[r] / MEV
            X.append(x)
            Y.append(cfg[sites].astype(np.float32))
    return np.concatenate(X)[:n_rows], np.concatenate(Y)[:n_rows]


def ess_per_second(result) -> tuple:
    """(ESS/s, per-point ESS, per-point max tau_int) of a PT/run_mc result:
    ESS = n_meas / (1 + 2 max(tau_int(E), tau_int(|m|))) summed over the points
    (the reference's tau_int convention, binning.jl:120-128), over the measurement
    phase's wall time."""
    ess, taus = [], []
    for p in result.points:
        t = max(float(np.nanmax(p.stats["energy"].tau_int)), float(np.nanmax(p.stats["absm"].tau_int)), 0.0)
        n = p.stats["energy"].count
        taus.append(t)
        ess.append(n / (1.0 + 2.0 * t))
    return float(np.sum(ess) / result.extra["measure_s"]), np.asarray(ess), np.asarray(taus)
