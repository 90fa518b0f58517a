"""Host-side statistics of a run: streaming log-binning, bin stores, jackknife and
the standard observables/evaluables (src/binning.jl:13-218,
src/observables.jl:85-249), fed by the measurement records the device writes
(one row per measurement and rung: E, m over active sites, sublattice sums).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MIN_BINS = 32     # binning.jl:13
MAX_LEVELS = 62   # binning.jl:14


class LogBinner:
    """Logarithmic binning accumulator (binning.jl:25-79). `push_many` feeds a
    batch of measurements and is equivalent to pushing them one at a time."""

    def __init__(self, ncomp: int):
        if ncomp < 1:
            raise ValueError(f"ncomp must be ≥ 1; got {ncomp}")
        self.ncomp = ncomp
        self.count = np.zeros(MAX_LEVELS, np.int64)
        self.sums = np.zeros((MAX_LEVELS, ncomp))
        self.sums2 = np.zeros((MAX_LEVELS, ncomp))
        self.pending = np.zeros((MAX_LEVELS, ncomp))
        self.pending_full = np.zeros(MAX_LEVELS, bool)
        self.n = 0

    def push(self, x):
        self.push_many(np.asarray(x, dtype=np.float64).reshape(1, self.ncomp))

    def state(self, prefix: str) -> dict:
        """Checkpoint arrays (the accs/<obs>/binner block of the checkpoint schema)."""
        return {prefix + "count": self.count.copy(), prefix + "sums": self.sums.copy(),
                prefix + "sums2": self.sums2.copy(), prefix + "pending": self.pending.copy(),
                prefix + "pending_full": self.pending_full.copy(), prefix + "n": np.array([self.n], np.int64)}

    def load_state(self, prefix: str, d) -> None:
        self.count = np.array(d[prefix + "count"], np.int64)
        self.sums = np.array(d[prefix + "sums"], np.float64)
        self.sums2 = np.array(d[prefix + "sums2"], np.float64)
        self.pending = np.array(d[prefix + "pending"], np.float64)
        self.pending_full = np.array(d[prefix + "pending_full"], bool)
        self.n = int(d[prefix + "n"][0])
        if self.sums.shape != (MAX_LEVELS, self.ncomp):
            raise ValueError("checkpointed LogBinner has another shape")

    def push_many(self, xs: np.ndarray):
        xs = np.asarray(xs, dtype=np.float64).reshape(-1, self.ncomp)
        if len(xs) == 0:
            return
        self.n += len(xs)
        stream = xs
        for k in range(MAX_LEVELS):
            if len(stream) == 0:
                break
            self.count[k] += len(stream)
            # sequential sums, as the one-at-a-time cascade accumulates them
            self.sums[k] = np.cumsum(np.vstack([self.sums[k], stream]), axis=0)[-1]
            self.sums2[k] = np.cumsum(np.vstack([self.sums2[k], stream * stream]), axis=0)[-1]
            seq = np.vstack([self.pending[k][None, :], stream]) if self.pending_full[k] else stream
            npairs = len(seq) // 2
            nxt = 0.5 * (seq[0:2 * npairs:2] + seq[1:2 * npairs:2])
            if len(seq) % 2 == 1:
                self.pending[k] = seq[-1]
                self.pending_full[k] = True
            else:
                self.pending_full[k] = False
            stream = nxt

    def mean(self):
        return np.full(self.ncomp, np.nan) if self.n == 0 else self.sums[0] / self.n

    def _level_error(self, k, j):
        n = self.count[k]
        if n < 2:
            return np.nan
        var = (self.sums2[k, j] - self.sums[k, j] ** 2 / n) / (n - 1)
        return np.sqrt(max(var, 0.0) / n)

    def _plateau(self):
        idx = np.nonzero(self.count >= MIN_BINS)[0]
        return int(idx[-1]) if len(idx) else 0

    def std_error(self):
        if self.n < 2:
            return np.full(self.ncomp, np.nan)
        k = self._plateau()
        return np.array([self._level_error(k, j) for j in range(self.ncomp)])

    def tau_int(self):
        if self.n < 2:
            return np.full(self.ncomp, np.nan)
        k = self._plateau()
        out = []
        for j in range(self.ncomp):
            e1 = self._level_error(0, j)
            out.append(0.5 * ((self._level_error(k, j) / e1) ** 2 - 1) if e1 > 0 else np.nan)
        return np.array(out)


class BinStore:
    """Fixed-layout bin means for jackknifing (binning.jl:138-188)."""

    def __init__(self, ncomp: int, bin_size: int, nbins: int):
        if ncomp < 1 or bin_size < 1 or nbins < 2:
            raise ValueError("BinStore needs ncomp ≥ 1, bin_size ≥ 1, nbins ≥ 2")
        self.ncomp, self.bin_size, self.nbins = ncomp, bin_size, nbins
        self.means = np.zeros((nbins, ncomp))
        self.nfull = 0
        self.acc = np.zeros(ncomp)
        self.nacc = 0

    def push_many(self, xs):
        for x in np.asarray(xs, dtype=np.float64).reshape(-1, self.ncomp):
            if self.nfull >= self.nbins:
                return
            self.acc += x
            self.nacc += 1
            if self.nacc == self.bin_size:
                self.means[self.nfull] = self.acc / self.bin_size
                self.nfull += 1
                self.acc[:] = 0.0
                self.nacc = 0

    def bin_means(self):
        return self.means[: self.nfull].copy()

    def state(self, prefix: str) -> dict:
        """Checkpoint arrays (the accs/<obs>/store block of the checkpoint schema)."""
        return {prefix + "means": self.means.copy(), prefix + "acc": self.acc.copy(),
                prefix + "ints": np.array([self.bin_size, self.nbins, self.nfull, self.nacc], np.int64)}

    def load_state(self, prefix: str, d) -> None:
        bs, nb, self.nfull, self.nacc = (int(x) for x in d[prefix + "ints"])
        if (bs, nb) != (self.bin_size, self.nbins):
            raise ValueError("checkpointed BinStore has another bin layout")
        self.means = np.array(d[prefix + "means"], np.float64).reshape(self.nbins, self.ncomp)
        self.acc = np.array(d[prefix + "acc"], np.float64).reshape(self.ncomp)


def jackknife(f, cols):
    """Leave-one-bin-out jackknife (binning.jl:198-218) -> (estimate, error)."""
    if not cols:
        raise ValueError("jackknife needs at least one input series")
    nb = len(cols[0])
    if any(len(c) != nb for c in cols):
        raise ValueError("jackknife input series have unequal lengths")
    if nb < 2:
        raise ValueError(f"jackknife needs ≥ 2 bins; got {nb}")
    tot = [float(np.sum(c)) for c in cols]
    full = f(*[t / nb for t in tot])
    th = np.array([f(*[(t - c[i]) / (nb - 1) for t, c in zip(tot, cols)]) for i in range(nb)])
    tbar = th.mean()
    return nb * full - (nb - 1) * tbar, float(np.sqrt((nb - 1) / nb * np.sum((th - tbar) ** 2)))


@dataclass
class ObservableStat:
    name: str
    mean: np.ndarray
    err: np.ndarray
    tau_int: np.ndarray
    count: int


@dataclass
class TempResult:
    """One temperature's results (src/run.jl:63-71)."""

    kT: float
    temperature: float
    stats: dict
    acceptance_metropolis: float
    acceptance_or: float
    final_step: float
    max_drift: float


@dataclass
class PTResult:
    """Result of a ladder / temperature batch (src/pt.jl PTResult)."""

    points: list
    swap_acceptance: np.ndarray
    final_configs: list
    seed: int
    extra: dict = field(default_factory=dict)


class StandardAccumulators:
    """The standard observables of one rung (observables.jl:85-92) accumulated
    from device records {E, m_x, m_y, m_z, sub_x1, sub_y1, sub_z1, ...}."""

    def __init__(self, n_cell_atoms: int, planned: int, nbins: int = 32):
        self.A = n_cell_atoms
        bs = max(1, planned // nbins)
        self.names = [("energy", 1), ("energy2", 1), ("m", 3), ("absm", 1), ("m2", 1), ("m4", 1),
                      ("sublattice_m", 3 * n_cell_atoms)]
        self.binners = {n: LogBinner(c) for n, c in self.names}
        self.stores = {n: BinStore(c, bs, nbins) for n, c in self.names}

    def state(self, prefix: str) -> dict:
        d = {}
        for n, _ in self.names:
            d.update(self.binners[n].state(f"{prefix}{n}/binner/"))
            d.update(self.stores[n].state(f"{prefix}{n}/store/"))
        return d

    def load_state(self, prefix: str, d) -> None:
        for n, _ in self.names:
            self.binners[n].load_state(f"{prefix}{n}/binner/", d)
            self.stores[n].load_state(f"{prefix}{n}/store/", d)

    def push_records(self, rec: np.ndarray):
        rec = np.asarray(rec, dtype=np.float64)
        E = rec[:, 0]
        m = rec[:, 1:4]
        m2 = np.sum(m * m, axis=1)
        vals = {"energy": E[:, None], "energy2": (E * E)[:, None], "m": m, "absm": np.sqrt(m2)[:, None],
                "m2": m2[:, None], "m4": (m2 * m2)[:, None], "sublattice_m": rec[:, 4:4 + 3 * self.A]}
        for n, _ in self.names:
            self.binners[n].push_many(vals[n])
            self.stores[n].push_many(vals[n])

    def finalize(self, kT: float, n_active: int) -> dict:
        """_finalize_stats (observables.jl:207-249) with the standard evaluables."""
        stats = {}
        for n, _ in self.names:
            b = self.binners[n]
            stats[n] = ObservableStat(n, b.mean(), b.std_error(), b.tau_int(), b.n)
        evals = [("specific_heat", ["energy", "energy2"], lambda e, e2: (e2 - e * e) / (n_active * kT * kT)),
                 ("susceptibility", ["m2", "absm"], lambda m2, am: n_active * (m2 - am * am) / kT),
                 ("binder", ["m2", "m4"], lambda m2, m4: m4 / (m2 * m2))]
        for name, inputs, f in evals:
            cols = [self.stores[i].bin_means()[:, 0] for i in inputs]
            if min(len(c) for c in cols) < 2:
                stats[name] = ObservableStat(name, np.array([np.nan]), np.array([np.nan]), np.array([np.nan]), 0)
                continue
            est, err = jackknife(f, cols)
            stats[name] = ObservableStat(name, np.array([est]), np.array([err]), np.array([np.nan]), len(cols[0]))
        return stats
