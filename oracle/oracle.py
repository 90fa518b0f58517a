"""ctypes binding of the FP64 oracle — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use this
module, and only as the checker or the timed CPU baseline. It builds its own
tables from a term list (an independent restatement of src/hamiltonian.jl) and
never touches libscemc_cuda.so.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

I32P = C.POINTER(C.c_int32)
U32P = C.POINTER(C.c_uint32)
F64P = C.POINTER(C.c_double)
I64P = C.POINTER(C.c_int64)
U8P = C.POINTER(C.c_uint8)

_lib = None


def build() -> pathlib.Path:
    src = HERE / "oracle.cpp"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        sig = {
            "or_last_error": (C.c_char_p, []),
            "or_philox4x32": (None, [U32P, C.c_uint32, C.c_uint32, U32P]),
            "or_philox_block": (None, [C.c_uint64, C.c_int32, C.c_int32, C.c_uint32, C.c_uint32, U32P]),
            "or_philox_uniform": (C.c_double, [C.c_uint32, C.c_uint32]),
            "or_philox_normal2": (None, [U32P, F64P]),
            "or_keyed_proposal": (None, [C.c_uint64, C.c_int32, C.c_int32, F64P, C.c_double, F64P, F64P]),
            "or_rotate": (None, [F64P, F64P, C.c_double, F64P]),
            "or_zlm_row": (None, [C.c_int, F64P, F64P]),
            "or_grad_zlm_row": (None, [C.c_int, F64P, F64P]),
            "or_energy_gradient": (None, [C.c_void_p, F64P, F64P]),
            "or_cpow": (None, [C.c_double, C.c_double, C.c_int, F64P]),
            "or_ham_build": (C.c_void_p, [C.c_int, C.c_int, F64P, I32P, I32P, I32P, I32P, F64P, I32P, F64P, F64P]),
            "or_ham_free": (None, [C.c_void_p]),
            "or_ham_scalar": (C.c_int64, [C.c_void_p, C.c_char_p]),
            "or_ham_array": (C.c_int64, [C.c_void_p, C.c_char_p, C.c_void_p, C.POINTER(C.c_int)]),
            "or_zrows": (None, [C.c_void_p, F64P, F64P]),
            "or_total_energy": (C.c_double, [C.c_void_p, F64P]),
            "or_total_energy_ref": (C.c_double, [C.c_void_p, F64P]),
            "or_site_coeffs": (None, [C.c_void_p, C.c_int, F64P, F64P]),
            "or_site_coeffs_ref": (None, [C.c_void_p, C.c_int, F64P, F64P]),
            "or_delta_energy": (C.c_double, [C.c_int, F64P, F64P, F64P]),
            "or_entry_walk_partial": (C.c_double, [C.c_void_p, F64P, F64P, C.c_int, C.c_int, C.c_int]),
            "or_keyed_sweep": (C.c_int, [C.c_void_p, F64P, F64P, F64P, I32P, C.c_double, C.c_double, C.c_uint64,
                                         C.c_int32, C.c_int]),
            "or_reduce_dE": (C.c_double, [C.c_void_p, F64P]),
            "or_swap_accepts": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
            "or_adapt_step": (C.c_double, [C.c_double, C.c_int64, C.c_int64, C.c_double]),
            "or_replay_sweep": (None, [C.c_void_p, F64P, F64P, F64P, U8P, C.c_double, F64P, F64P, U8P, F64P]),
            "or_chain_new": (C.c_void_p, [C.c_void_p, F64P, C.c_uint64, C.c_double]),
            "or_chain_free": (None, [C.c_void_p]),
            "or_chain_get": (None, [C.c_void_p, F64P, F64P, I64P, I64P, F64P]),
            "or_chain_sweeps": (None, [C.c_void_p, C.c_void_p, C.c_double, C.c_int64, C.c_int, C.c_int]),
            "or_chain_renormalize": (C.c_double, [C.c_void_p, C.c_void_p]),
            "or_stats_len": (C.c_int, [C.c_void_p]),
            "or_run_mc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                    C.c_double, C.c_int64, C.c_int64, C.c_int, C.c_int, F64P]),
            "or_run_pt": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), F64P, C.c_int64, C.c_int64,
                                    C.c_int64, C.c_int64, C.c_int, C.c_double, C.c_int64, C.c_int64, C.c_int,
                                    C.c_uint64, C.c_int, F64P, I64P, I64P]),
            "or_logbinner_stats": (None, [F64P, C.c_int64, F64P, F64P, F64P]),
            "or_kb_ev": (C.c_double, []),
            "or_mu_b_ev_t": (C.c_double, []),
            "or_max_threads": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def philox4x32(ctr, key):
    out = np.zeros(4, np.uint32)
    c = np.asarray(ctr, dtype=np.uint32)
    lib().or_philox4x32(_p(c, C.c_uint32), C.c_uint32(key[0]), C.c_uint32(key[1]), _p(out, C.c_uint32))
    return tuple(int(x) for x in out)


def philox_block(seed, site, sweep, slot, tag=0):
    out = np.zeros(4, np.uint32)
    lib().or_philox_block(C.c_uint64(seed), site, sweep, slot, tag, _p(out, C.c_uint32))
    return tuple(int(x) for x in out)


def grad_zlm_row(lmax, u):
    """Tangent gradients of the tesseral row at u: ((lmax+1)^2, 3)."""
    uu = np.ascontiguousarray(u, dtype=np.float64)
    g = np.zeros(((lmax + 1) ** 2, 3))
    lib().or_grad_zlm_row(int(lmax), _p(uu, C.c_double), _p(g, C.c_double))
    return g


def philox_uniform(hi, lo):
    return lib().or_philox_uniform(hi, lo)


def philox_normal2(blk):
    b = np.asarray(blk, dtype=np.uint32)
    out = np.zeros(2)
    lib().or_philox_normal2(_p(b, C.c_uint32), _p(out, C.c_double))
    return float(out[0]), float(out[1])


def keyed_proposal(seed, site, sweep, e, step):
    e = np.ascontiguousarray(e, dtype=np.float64)
    e2 = np.zeros(3)
    u = C.c_double()
    lib().or_keyed_proposal(C.c_uint64(seed), site, sweep, _p(e, C.c_double), step, _p(e2, C.c_double), C.byref(u))
    return e2, u.value


def rotate(e, axis, th):
    e = np.ascontiguousarray(e, dtype=np.float64)
    a = np.ascontiguousarray(axis, dtype=np.float64)
    out = np.zeros(3)
    lib().or_rotate(_p(e, C.c_double), _p(a, C.c_double), th, _p(out, C.c_double))
    return out


def zlm_row(lmax, u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros((lmax + 1) ** 2)
    lib().or_zlm_row(lmax, _p(u, C.c_double), _p(out, C.c_double))
    return out


def cpow(z, p):
    out = np.zeros(2)
    lib().or_cpow(z.real, z.imag, p, _p(out, C.c_double))
    return complex(out[0], out[1])


def adapt_step(step, acc, att, target=0.5):
    """The step after one adaptation window with acc of att Metropolis moves accepted
    (updates.jl:296-305)."""
    return lib().or_adapt_step(float(step), int(acc), int(att), float(target))


def swap_accepts(kt_a, kt_b, E_a, E_b, u):
    return bool(lib().or_swap_accepts(kt_a, kt_b, E_a, E_b, u))


def logbinner_stats(xs):
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    m, e, t = C.c_double(), C.c_double(), C.c_double()
    lib().or_logbinner_stats(_p(xs, C.c_double), len(xs), C.byref(m), C.byref(e), C.byref(t))
    return m.value, e.value, t.value


_DT = {0: np.int32, 1: np.int8, 2: np.uint8, 3: np.float64}


class OracleHamiltonian:
    """The oracle's own TiledHamiltonian, built from a term list (objects with
    coef, atoms, shifts, ls, folded attributes)."""

    def __init__(self, n_cell_atoms, terms, dims=(1, 1, 1), magmoms=None, field=None):
        coef, body, atoms, shifts, ls, folded = [], [], [], [], [], []
        for t in terms:
            coef.append(float(t.coef))
            body.append(len(t.atoms))
            atoms += [int(a) for a in t.atoms]
            for s in t.shifts:
                shifts += [int(x) for x in s]
            ls += [int(l) for l in t.ls]
            folded += list(np.asarray(t.folded, dtype=np.float64).ravel(order="F"))
        arrs = [np.asarray(coef, np.float64), np.asarray(body, np.int32), np.asarray(atoms, np.int32),
                np.asarray(shifts, np.int32), np.asarray(ls, np.int32), np.asarray(folded, np.float64)]
        arrs = [a if a.size else np.zeros(1, a.dtype) for a in arrs]
        d = np.asarray(dims, np.int32)
        mm = None if magmoms is None else np.asarray(magmoms, np.float64)
        fl = None if field is None else np.asarray(field, np.float64)
        self._keep = (arrs, d, mm, fl)
        h = lib().or_ham_build(n_cell_atoms, len(coef), _p(arrs[0], C.c_double), _p(arrs[1], C.c_int32),
                               _p(arrs[2], C.c_int32), _p(arrs[3], C.c_int32), _p(arrs[4], C.c_int32),
                               _p(arrs[5], C.c_double), _p(d, C.c_int32),
                               None if mm is None else _p(mm, C.c_double),
                               None if fl is None else _p(fl, C.c_double))
        if not h:
            raise ValueError(lib().or_last_error().decode())
        self.h = C.c_void_p(h)
        for k in ["n_sites", "nlm", "lmax", "n_colors", "n_active", "n_cell_atoms", "n_terms", "n_fitted"]:
            setattr(self, k, int(lib().or_ham_scalar(self.h, k.encode())))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_ham_free(self.h)
            self.h = None

    def array(self, name):
        code = C.c_int()
        n = lib().or_ham_array(self.h, name.encode(), None, C.byref(code))
        if n < 0:
            raise KeyError(name)
        out = np.zeros(max(n, 0), dtype=_DT[code.value])
        if n > 0:
            lib().or_ham_array(self.h, name.encode(), out.ctypes.data_as(C.c_void_p), C.byref(code))
        return out

    # energy contract ------------------------------------------------------
    def zrows(self, config):
        cfg = np.ascontiguousarray(config, dtype=np.float64).reshape(self.n_sites, 3)
        z = np.zeros((self.n_sites, self.nlm))
        lib().or_zrows(self.h, _p(cfg, C.c_double), _p(z, C.c_double))
        return z

    def total_energy_rows(self, zrows):
        z = np.ascontiguousarray(zrows, dtype=np.float64)
        return lib().or_total_energy(self.h, _p(z, C.c_double))

    def total_energy(self, config):
        return self.total_energy_rows(self.zrows(config))

    def total_energy_ref(self, config):
        z = self.zrows(config)
        return lib().or_total_energy_ref(self.h, _p(z, C.c_double))

    def energy_gradient(self, config):
        """All-site tangent gradient G[s] = sum_t c_t(s) grad Z_t(e_s) (n_sites x 3)."""
        cfg = np.ascontiguousarray(config, dtype=np.float64).reshape(self.n_sites, 3)
        G = np.zeros((self.n_sites, 3))
        lib().or_energy_gradient(self.h, _p(cfg, C.c_double), _p(G, C.c_double))
        return G

    def site_coeffs(self, s, zrows, ref=False):
        z = np.ascontiguousarray(zrows, dtype=np.float64)
        c = np.zeros(self.nlm)
        fn = lib().or_site_coeffs_ref if ref else lib().or_site_coeffs
        fn(self.h, int(s), _p(z, C.c_double), _p(c, C.c_double))
        return c

    def delta_energy(self, c, zold, znew):
        c = np.ascontiguousarray(c, dtype=np.float64)
        a = np.ascontiguousarray(zold, dtype=np.float64)
        b = np.ascontiguousarray(znew, dtype=np.float64)
        return lib().or_delta_energy(self.nlm, _p(c, C.c_double), _p(a, C.c_double), _p(b, C.c_double))

    def entry_walk_partial(self, zrows, znew, s, lane, ws):
        z = np.ascontiguousarray(zrows, dtype=np.float64)
        zn = np.ascontiguousarray(znew, dtype=np.float64)
        return lib().or_entry_walk_partial(self.h, _p(z, C.c_double), _p(zn, C.c_double), s, lane, ws)

    def keyed_sweep(self, config, zrows, beta, step, seed, sweep, ws=32):
        """One _metropolis_sweep_keyed_ref! sweep in place; returns (nacc, dE, acc)."""
        dE = np.zeros(self.n_sites)
        acc = np.zeros(self.n_sites, np.int32)
        n = lib().or_keyed_sweep(self.h, _p(config, C.c_double), _p(zrows, C.c_double), _p(dE, C.c_double),
                                 _p(acc, C.c_int32), beta, step, C.c_uint64(seed), sweep, ws)
        return n, dE, acc

    def reduce_dE(self, dE):
        dE = np.ascontiguousarray(dE, dtype=np.float64)
        return lib().or_reduce_dE(self.h, _p(dE, C.c_double))

    def replay_sweep(self, config, prop, u, dev_acc, beta, want_c=False):
        """Replays one device sweep (see oracle.cpp or_replay_sweep). config is updated
        in place with the device's decisions. Returns (dE64, scale, oracle_accept, c)."""
        cfg = np.ascontiguousarray(config, dtype=np.float64)
        pr = np.ascontiguousarray(prop, dtype=np.float64)
        uu = np.ascontiguousarray(u, dtype=np.float64)
        da = np.ascontiguousarray(dev_acc, dtype=np.uint8)
        dE = np.zeros(self.n_sites)
        sc = np.zeros(self.n_sites)
        oa = np.zeros(self.n_sites, np.uint8)
        cc = np.zeros((self.n_sites, self.nlm)) if want_c else None
        lib().or_replay_sweep(self.h, _p(cfg, C.c_double), _p(pr, C.c_double), _p(uu, C.c_double),
                              _p(da, C.c_uint8), beta, _p(dE, C.c_double), _p(sc, C.c_double), _p(oa, C.c_uint8),
                              None if cc is None else _p(cc, C.c_double))
        config[...] = cfg.reshape(np.shape(config))
        return dE, sc, oa.astype(bool), cc

    def stats_len(self):
        return lib().or_stats_len(self.h)


class OracleChain:
    """A keyed-RNG CPU chain (the timed baseline and the statistics oracle)."""

    def __init__(self, H: OracleHamiltonian, config, seed, step=0.6):
        self.H = H
        cfg = np.ascontiguousarray(config, dtype=np.float64).reshape(H.n_sites, 3)
        self.c = C.c_void_p(lib().or_chain_new(H.h, _p(cfg, C.c_double), C.c_uint64(seed), step))

    def __del__(self):
        if getattr(self, "c", None) and _lib is not None:
            _lib.or_chain_free(self.c)
            self.c = None

    def get(self):
        cfg = np.zeros((self.H.n_sites, 3))
        E = C.c_double()
        sw = C.c_int64()
        cnt = np.zeros(4, np.int64)
        st = C.c_double()
        lib().or_chain_get(self.c, _p(cfg, C.c_double), C.byref(E), C.byref(sw), _p(cnt, C.c_int64), C.byref(st))
        return cfg, E.value, sw.value, cnt, st.value

    def sweeps(self, beta, n, n_or=0, threads=1):
        lib().or_chain_sweeps(self.H.h, self.c, beta, n, n_or, threads)

    def renormalize(self):
        return lib().or_chain_renormalize(self.H.h, self.c)

    def run_mc(self, kT, sweeps_therm, sweeps_measure, measure_interval=1, n_or=0, adapt_target=0.5,
               adapt_interval=50, renorm_interval=1000, nbins=32, threads=1):
        out = np.zeros(self.H.stats_len())
        lib().or_run_mc(self.H.h, self.c, kT, sweeps_therm, sweeps_measure, measure_interval, n_or, adapt_target,
                        adapt_interval, renorm_interval, nbins, threads, _p(out, C.c_double))
        return unpack_stats(self.H, out)


def run_pt(H: OracleHamiltonian, chains, kts, sweeps_therm, sweeps_measure, measure_interval=1,
           exchange_interval=10, n_or=0, adapt_target=0.5, adapt_interval=50, renorm_interval=1000, nbins=32,
           exchange_seed=0x5CE3C0FFEE5EED, threads=1):
    R = len(chains)
    arr = (C.c_void_p * R)(*[c.c for c in chains])
    kt = np.ascontiguousarray(kts, dtype=np.float64)
    L = H.stats_len()
    out = np.zeros(R * L)
    att = np.zeros(R, np.int64)
    acc = np.zeros(R, np.int64)
    lib().or_run_pt(H.h, R, arr, _p(kt, C.c_double), sweeps_therm, sweeps_measure, measure_interval,
                    exchange_interval, n_or, adapt_target, adapt_interval, renorm_interval, nbins,
                    C.c_uint64(exchange_seed), threads, _p(out, C.c_double), _p(att, C.c_int64), _p(acc, C.c_int64))
    pts = [unpack_stats(H, out[r * L:(r + 1) * L]) for r in range(R)]
    with np.errstate(invalid="ignore", divide="ignore"):
        swaps = acc[:R - 1] / att[:R - 1]
    return pts, swaps


def unpack_stats(H, out):
    """Stats block -> dict name -> (mean[], err[], tau[]) plus evaluables and scalars."""
    names = [("energy", 1), ("energy2", 1), ("m", 3), ("absm", 1), ("m2", 1), ("m4", 1),
             ("sublattice_m", 3 * H.n_cell_atoms)]
    res = {}
    w = 0
    for name, nc in names:
        blk = np.asarray(out[w:w + 3 * nc]).reshape(nc, 3)
        res[name] = (blk[:, 0].copy(), blk[:, 1].copy(), blk[:, 2].copy())
        w += 3 * nc
    for name in ("specific_heat", "susceptibility", "binder"):
        res[name] = (np.array([out[w]]), np.array([out[w + 1]]), np.array([np.nan]))
        w += 2
    res["acceptance_metropolis"] = out[w]
    res["acceptance_or"] = out[w + 1]
    res["final_step"] = out[w + 2]
    res["max_drift"] = out[w + 3]
    return res
