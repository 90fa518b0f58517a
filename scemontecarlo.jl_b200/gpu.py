"""The reference's device-path API over libscemc_cuda.so.

Names, argument meaning and error behaviour follow src/gpu/*.jl:
  GPUTiledHamiltonian  gpu_hamiltonian.jl:61-88
  GPUChainState        gpu_state.jl:19-61
  gpu_metropolis_sweep gpu_sweep.jl:158-190
  gpu_run_sweeps       gpu_sweep.jl:204-218
  to_host / from_host  gpu_state.jl:71-86
  swap_payload         gpu_pt.jl:46-51
  gpu_run_pt           gpu_pt.jl:261-316
plus the device overrelaxation sweep (the reference has it on the CPU only,
src/updates.jl:231-248) and the batched ensemble the PT driver runs on.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .hamiltonian import KB_EV, TiledHamiltonian, resolve_kt
from .stats import PTResult, StandardAccumulators, TempResult

check = _lib.check
ptr = _lib.ptr


def _ispow2(n: int) -> bool:
    return n >= 1 and (n & (n - 1)) == 0


class GPUTiledHamiltonian:
    """Device tables of one TiledHamiltonian (the 'backend' is the current CUDA device)."""

    def __init__(self, H: TiledHamiltonian):
        if H.lmax > 6:
            raise ValueError(f"lmax = {H.lmax} unsupported on the device path (gated ≤ 6)")
        self.host = H
        d = H.desc()
        h = C.c_void_p()
        check(_lib.lib().scemc_tables_create(C.byref(d), C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) and _lib._lib is not None:
            _lib._lib.scemc_tables_destroy(self.h)
            self.h = None

    @property
    def n_sites(self) -> int:
        return self.host.n_sites

    def stats(self):
        """(mean distinct neighbours d, mean adjacency entries A, device table bytes)."""
        dm, am, by = C.c_double(), C.c_double(), C.c_int64()
        check(_lib.lib().scemc_tables_stats(self.h, C.byref(dm), C.byref(am), C.byref(by)))
        return dm.value, am.value, by.value

    def records_per_site(self) -> float:
        """Mean merged records per active site that the fast kernels walk."""
        r = C.c_double()
        check(_lib.lib().scemc_tables_records(self.h, C.byref(r)))
        return r.value


@dataclass
class ChainState:
    """Host mirror of a chain (the fields of src/state.jl:17-46 the device path uses)."""

    config: np.ndarray  # (n_sites, 3) FP64
    energy: float
    step: float = 0.6
    acc_metro: int = 0
    att_metro: int = 0
    acc_or: int = 0
    att_or: int = 0
    max_drift: float = 0.0


def _config_array(config, n_sites: int) -> np.ndarray:
    a = np.ascontiguousarray(config, dtype=np.float64).reshape(-1)
    if a.size != 3 * n_sites:
        raise ValueError(f"config has {a.size // 3} sites; expected {n_sites}")
    return a


class GPUChainState:
    """Device chain: FP32 float4 spins + FP64 running energy; seed, sweep index,
    step and counters stay with the object (the lane)."""

    def __init__(self, gH: GPUTiledHamiltonian, st, seed: int, step: Optional[float] = None,
                 energy: Optional[float] = None):
        if isinstance(st, ChainState):
            config, energy0, step0 = st.config, st.energy, st.step
        else:
            config, energy0, step0 = st, None, 0.6
        if step is not None:
            step0 = step
        if energy is not None:
            energy0 = energy
        self.gH = gH
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        cfg = _config_array(config, gH.n_sites)
        h = C.c_void_p()
        check(_lib.lib().scemc_chain_create(gH.h, ptr(cfg, C.c_double), 0.0 if energy0 is None else float(energy0),
                                            C.c_uint64(self.seed), float(step0), C.byref(h)))
        self.h = h
        if energy0 is None:  # anchor on the FP64 energy of the stored (FP32) spins
            check(_lib.lib().scemc_renormalize(self.h, None))

    def __del__(self):
        if getattr(self, "h", None) and _lib._lib is not None:
            _lib._lib.scemc_chain_destroy(self.h)
            self.h = None

    @property
    def energy(self) -> float:
        e = C.c_double()
        check(_lib.lib().scemc_download(self.h, None, C.byref(e), None, None))
        return e.value

    @property
    def sweep_index(self) -> int:
        s = C.c_int64()
        check(_lib.lib().scemc_download(self.h, None, None, C.byref(s), None))
        return s.value

    def counters(self):
        c = np.zeros(4, np.int64)
        check(_lib.lib().scemc_download(self.h, None, None, None, ptr(c, C.c_int64)))
        return c

    def set_step(self, step: float):
        check(_lib.lib().scemc_set_step(self.h, float(step)))

    def total_energy(self) -> float:
        """FP64 full recompute of the device state (does not touch the running energy)."""
        e = C.c_double()
        check(_lib.lib().scemc_total_energy(self.h, 0, C.byref(e)))
        return e.value

    def renormalize(self) -> float:
        d = np.zeros(1)
        check(_lib.lib().scemc_renormalize(self.h, ptr(d, C.c_double)))
        return float(d[0])


def gpu_metropolis_sweep(gst: GPUChainState, gH: GPUTiledHamiltonian, beta: float, workgroupsize: int = 128) -> int:
    """One device Metropolis sweep; returns the number of accepted moves."""
    if not _ispow2(int(workgroupsize)):
        raise ValueError(f"workgroupsize must be a power of two (got {workgroupsize})")
    n = C.c_int64()
    check(_lib.lib().scemc_metropolis_sweep(gst.h, gH.h, float(beta), int(workgroupsize), C.byref(n)))
    return n.value


def gpu_overrelaxation_sweep(gst: GPUChainState, gH: GPUTiledHamiltonian, beta: float,
                             workgroupsize: int = 128):
    """One device overrelaxation sweep; returns (accepted, attempted)."""
    if not _ispow2(int(workgroupsize)):
        raise ValueError(f"workgroupsize must be a power of two (got {workgroupsize})")
    a, t = C.c_int64(), C.c_int64()
    check(_lib.lib().scemc_overrelaxation_sweep(gst.h, gH.h, float(beta), int(workgroupsize), C.byref(a),
                                                C.byref(t)))
    return a.value, t.value


def to_host(st: ChainState, gst: GPUChainState) -> ChainState:
    cfg = np.zeros(3 * gst.gH.n_sites)
    e = C.c_double()
    check(_lib.lib().scemc_download(gst.h, ptr(cfg, C.c_double), C.byref(e), None, None))
    st.config = cfg.reshape(-1, 3)
    st.energy = e.value
    return st


def from_host(gst: GPUChainState, st: ChainState) -> GPUChainState:
    cfg = _config_array(st.config, gst.gH.n_sites)
    check(_lib.lib().scemc_upload(gst.h, ptr(cfg, C.c_double), float(st.energy)))
    return gst


def gpu_energy_gradient(gH: GPUTiledHamiltonian, config) -> np.ndarray:
    """All-site energy gradient (gpu_energy_gradient!, gpu_gradient.jl:193-231): the
    tangent gradient of the energy at every spin, (n_sites, 3) for one configuration
    or (R, n_sites, 3) for a stack of R configurations."""
    cfg = np.ascontiguousarray(config, np.float64)
    one = cfg.ndim == 2
    cfg = cfg.reshape(-1, gH.n_sites, 3)
    out = np.zeros_like(cfg)
    check(_lib.lib().scemc_energy_gradient(gH.h, ptr(cfg, C.c_double), cfg.shape[0], ptr(out, C.c_double)))
    return out[0] if one else out


def gpu_run_sweeps(gst: GPUChainState, gH: GPUTiledHamiltonian, st: ChainState, beta: float, nsweeps: int,
                   renorm_interval: int = 1000, workgroupsize: int = 128) -> GPUChainState:
    """nsweeps device Metropolis sweeps with a device renormalisation + FP64 recompute
    every renorm_interval sweeps (<= 0 disables); downloads the state into st."""
    if not _ispow2(int(workgroupsize)):
        raise ValueError(f"workgroupsize must be a power of two (got {workgroupsize})")
    check(_lib.lib().scemc_run_sweeps(gst.h, gH.h, float(beta), int(nsweeps), int(renorm_interval),
                                      int(workgroupsize)))
    to_host(st, gst)
    return gst


def swap_payload(a: GPUChainState, b: GPUChainState):
    check(_lib.lib().scemc_swap_payload(a.h, b.h))


class PinnedHost:
    """A float64 host buffer page-locked through scemc_host_register (released on
    close or exit of a `with` block): uploads from it and downloads into it are
    direct DMA."""

    def __init__(self, n: int):
        self.array = np.zeros(int(n))
        check(_lib.lib().scemc_host_register(self.array.ctypes.data, self.array.nbytes))
        self._pinned = True

    def close(self):
        if getattr(self, "_pinned", False):
            self._pinned = False
            check(_lib.lib().scemc_host_unregister(self.array.ctypes.data))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GPUBatch:
    """Replicas of one or more table sets advancing together (PT rungs, temperature
    sets, chains of uneven supercells). Slots are numbered table-major."""

    def __init__(self, gHs: Sequence[GPUTiledHamiltonian], replicas: Sequence[int], configs, seeds, steps,
                 energies=None):
        self.gHs = list(gHs)
        self.replicas = [int(r) for r in replicas]
        nslots = sum(self.replicas)
        cfg = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float64).reshape(-1) for c in configs]))
        exp = sum(3 * g.n_sites * r for g, r in zip(self.gHs, self.replicas))
        if cfg.size != exp:
            raise ValueError("configs do not match the table sizes")
        en = np.zeros(nslots) if energies is None else np.ascontiguousarray(energies, np.float64)
        sd = np.ascontiguousarray([int(s) & 0xFFFFFFFFFFFFFFFF for s in seeds], dtype=np.uint64)
        stp = np.ascontiguousarray(np.broadcast_to(np.asarray(steps, np.float64), (nslots,)))
        tabs = (C.c_void_p * len(self.gHs))(*[g.h for g in self.gHs])
        reps = np.ascontiguousarray(self.replicas, np.int32)
        h = C.c_void_p()
        check(_lib.lib().scemc_batch_create(len(self.gHs), tabs, ptr(reps, C.c_int32), ptr(cfg, C.c_double),
                                            ptr(en, C.c_double), ptr(sd, C.c_uint64), ptr(stp, C.c_double),
                                            C.byref(h)))
        self.h = h
        self.n_slots = nslots
        self.n_sites_total = exp // 3  # spins of every chain
        if energies is None:
            check(_lib.lib().scemc_renormalize(self.h, None))
            self.reset_counters()

    def __del__(self):
        if getattr(self, "h", None) and _lib._lib is not None:
            _lib._lib.scemc_batch_destroy(self.h)
            self.h = None

    def set_betas(self, betas):
        b = np.ascontiguousarray(betas, np.float64)
        check(_lib.lib().scemc_batch_set_betas(self.h, ptr(b, C.c_double)))

    def set_steps(self, steps):
        s = np.ascontiguousarray(np.broadcast_to(np.asarray(steps, np.float64), (self.n_slots,)))
        check(_lib.lib().scemc_batch_set_steps(self.h, ptr(s, C.c_double)))

    @staticmethod
    def params(nsweeps, or_per_metropolis=0, exchange=False, exchange_interval=1, adapt_interval=0,
               adapt_target=0.5, renorm_interval=0, measure_interval=0, lanes_per_site=0, mode=0, phase_done=0,
               phase_total=0, kernel=0, proposals=0, rep_replicas=0, rep_threads_per_item=0,
               rep_prefetch=0) -> _lib.RunParams:
        return _lib.RunParams(int(nsweeps), int(or_per_metropolis), int(bool(exchange)), int(exchange_interval),
                              int(adapt_interval), float(adapt_target), int(renorm_interval), int(measure_interval),
                              int(lanes_per_site), int(mode), int(phase_done), int(phase_total), int(kernel),
                              int(proposals), int(rep_replicas), int(rep_threads_per_item), int(rep_prefetch))

    def run(self, nsweeps, **kw):
        """Runs `nsweeps` compound sweeps (see scemc_run_params) and waits for them."""
        p = self.params(nsweeps, **kw)
        check(_lib.lib().scemc_batch_run(self.h, C.byref(p)))

    def run_async(self, p: _lib.RunParams):
        """Enqueues a run on the batch stream; call sync() before touching the batch."""
        check(_lib.lib().scemc_batch_run_async(self.h, C.byref(p)))

    def sync(self):
        check(_lib.lib().scemc_batch_sync(self.h))

    def stream(self) -> int:
        s = C.c_void_p()
        check(_lib.lib().scemc_batch_stream(self.h, C.byref(s)))
        return s.value or 0

    def upload(self, configs, energies=None):
        """Replaces every chain's spins (the payload of all chains, table-major, each
        3 x n_sites) and optionally the running energies. With energies=None the running
        energies keep their old values: pass the new configurations' energies, or call
        renormalize() after the upload (FP64 recompute), before relying on them."""
        cfg = np.ascontiguousarray(configs, np.float64).reshape(-1)
        if cfg.size != 3 * self.n_sites_total:
            raise ValueError("configs hold %d values, the batch %d" % (cfg.size, 3 * self.n_sites_total))
        en = None if energies is None else np.ascontiguousarray(energies, np.float64).reshape(-1)
        if en is not None and en.size != self.n_slots:
            raise ValueError("one energy per slot is needed")
        check(_lib.lib().scemc_batch_upload(self.h, ptr(cfg, C.c_double), None if en is None else ptr(en, C.c_double)))

    def save_state(self) -> np.ndarray:
        """The batch's mutable device state as a byte array (scemc_batch_save_state)."""
        n = C.c_int64()
        check(_lib.lib().scemc_batch_state_bytes(self.h, C.byref(n)))
        buf = np.zeros(n.value, np.uint8)
        check(_lib.lib().scemc_batch_save_state(self.h, buf.ctypes.data, buf.size))
        return buf

    def load_state(self, buf) -> None:
        """Restores a state saved from a batch of the same tables and replica counts."""
        buf = np.ascontiguousarray(buf, np.uint8)
        check(_lib.lib().scemc_batch_load_state(self.h, buf.ctypes.data, buf.size))

    def profile(self, on: bool):
        check(_lib.lib().scemc_batch_profile(self.h, int(bool(on))))

    def autotune(self, or_per_metropolis: int = 0, sweeps_per_trial: int = 5):
        """Times the launch forms on this batch (its chains advance) and keeps the
        fastest for runs with mode=0 and kernel=0; returns a dict with the chosen mode,
        proposals, lanes, kernel and its ms/sweep."""
        m, q, g, k, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        check(_lib.lib().scemc_batch_autotune(self.h, int(or_per_metropolis), int(sweeps_per_trial), C.byref(m),
                                              C.byref(q), C.byref(g), C.byref(k), C.byref(ms)))
        return {"mode": m.value, "proposals": q.value, "lanes": g.value, "kernel": k.value, "ms_per_sweep": ms.value}

    def set_learned(self, net, env) -> None:
        """Registers a learned proposal network (scemc.learned.ProposalNet, or None to
        unregister) with its environment table (n_sites x net.n_env per table,
        0-based); runs with proposals=3 then use it for every Metropolis proposal."""
        if net is None:
            check(_lib.lib().scemc_batch_set_learned(self.h, None, None, 14))
            self._net = None
            return
        if net.n_env == 0:  # field mode: the network reads the site coefficients
            check(_lib.lib().scemc_batch_set_learned(self.h, net.h, None, 0))
            self._net = net
            return
        tabs = env if isinstance(env, (list, tuple)) else [env]
        k = int(net.n_env)
        if any(np.asarray(e).reshape(-1).size != g.n_sites * k for e, g in zip(tabs, self.gHs)):
            raise ValueError(f"every environment table must be n_sites x {k}")
        env = np.ascontiguousarray(np.concatenate([np.asarray(e, np.int32).reshape(-1) for e in tabs]), np.int32)
        check(_lib.lib().scemc_batch_set_learned(self.h, net.h, ptr(env, C.c_int32), k))
        self._net = net  # the batch does not own the network: keep it alive

    def site_coeffs(self, slot: int) -> np.ndarray:
        """Leave-one-out coefficients (rows 1..NR) of every site of a slot's current
        spins, (n_sites, NR) float32 (scemc_batch_site_coeffs)."""
        li = 0
        off = 0
        for i, r in enumerate(self.replicas):
            if slot < off + r:
                li = i
                break
            off += r
        n = self.gHs[li].n_sites
        nr = 3 if self.gHs[li].host.lmax == 1 else 8
        out = np.zeros(n * nr, np.float32)
        check(_lib.lib().scemc_batch_site_coeffs(self.h, int(slot), ptr(out, C.c_float)))
        return out.reshape(n, nr)

    def fetch_record_ratio(self) -> np.ndarray:
        """log q(e|env) - log q(e'|env) of the recorded learned Metropolis pass."""
        out = np.zeros(self.gHs[getattr(self, "_rec_table", 0)].n_sites)
        check(_lib.lib().scemc_batch_fetch_record_ratio(self.h, ptr(out, C.c_double)))
        return out

    def launches(self) -> int:
        """Kernels this batch has enqueued (graph replays count their kernel nodes)."""
        n = C.c_int64()
        check(_lib.lib().scemc_batch_launches(self.h, C.byref(n)))
        return n.value

    def kernel_time(self):
        """(summed device ms of the sweep passes, number of passes) since profile(True)."""
        ms, n = C.c_double(), C.c_int64()
        check(_lib.lib().scemc_batch_kernel_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def renormalize(self):
        d = np.zeros(self.n_slots)
        check(_lib.lib().scemc_renormalize(self.h, ptr(d, C.c_double)))
        return d

    def reset_counters(self):
        check(_lib.lib().scemc_batch_reset_counters(self.h))

    def total_energy(self, slot: int) -> float:
        e = C.c_double()
        check(_lib.lib().scemc_total_energy(self.h, int(slot), C.byref(e)))
        return e.value

    def download(self, out=None):
        """The batch state. `out`, when given, is a C-contiguous float64 buffer of
        3 x (total spins) that receives the payload (pinned host memory makes the
        copy a direct DMA); the returned configs are views into it."""
        n = self.n_slots
        tot = self.n_sites_total
        if out is None:
            cfg = np.empty(3 * tot)
        else:
            cfg = out.reshape(-1)
            if cfg.dtype != np.float64 or cfg.size != 3 * tot or not cfg.flags.c_contiguous or not cfg.flags.writeable:
                raise ValueError("out must be a writeable C-contiguous float64 buffer of 3 x %d values" % tot)
        en = np.zeros(n)
        sor = np.zeros(n, np.int32)
        cnt = np.zeros(4 * n, np.int64)
        sw = np.zeros(2 * n, np.int64)
        st = np.zeros(n)
        md = np.zeros(n)
        check(_lib.lib().scemc_batch_download(self.h, ptr(cfg, C.c_double), ptr(en, C.c_double),
                                              ptr(sor, C.c_int32), ptr(cnt, C.c_int64), ptr(sw, C.c_int64),
                                              ptr(st, C.c_double), ptr(md, C.c_double)))
        configs, off = [], 0
        for g, r in zip(self.gHs, self.replicas):
            for _ in range(r):
                configs.append(cfg[off:off + 3 * g.n_sites].reshape(-1, 3))
                off += 3 * g.n_sites
        return dict(configs=configs, energies=en, slot_of_rung=sor, counters=cnt.reshape(n, 4),
                    swaps=sw.reshape(n, 2), steps=st, max_drift=md)

    def fetch_measurements(self):
        n = C.c_int64()
        rl = C.c_int32()
        check(_lib.lib().scemc_batch_fetch_measurements(self.h, None, 0, C.byref(n), C.byref(rl)))
        buf = np.zeros(max(1, n.value * self.n_slots * rl.value))
        check(_lib.lib().scemc_batch_fetch_measurements(self.h, ptr(buf, C.c_double), n.value, C.byref(n),
                                                        C.byref(rl)))
        return buf[: n.value * self.n_slots * rl.value].reshape(n.value, self.n_slots, rl.value)

    def record(self, on: bool):
        check(_lib.lib().scemc_batch_record(self.h, int(bool(on))))

    def record_slot(self, table: int = 0, replica: int = 0):
        """Chooses the recorded replica (0-based replica of 0-based table)."""
        check(_lib.lib().scemc_batch_record_slot(self.h, int(table), int(replica)))
        self._rec_table = int(table)

    def fetch_record(self, pass_: int = -1):
        """Recorded (proposal, u, dE32, flag) of the recorded replica for pass -1
        (Metropolis) or overrelaxation pass k."""
        n = self.gHs[getattr(self, "_rec_table", 0)].n_sites
        prop = np.zeros(3 * n, np.float32)
        u = np.zeros(n)
        dE = np.zeros(n, np.float32)
        acc = np.zeros(n, np.uint8)
        check(_lib.lib().scemc_batch_fetch_record(self.h, int(pass_), ptr(prop, C.c_float), ptr(u, C.c_double),
                                                  ptr(dE, C.c_float), ptr(acc, C.c_uint8)))
        return prop.reshape(n, 3), u, dE, acc


def _random_configs(n_sites: int, count: int, rng: np.random.Generator):
    out = []
    for _ in range(count):
        v = rng.standard_normal((n_sites, 3))
        out.append(v / np.linalg.norm(v, axis=1, keepdims=True))
    return out


def gpu_run_pt(gHs, *, temperature=None, kT=None, exchange: bool = True, exchange_interval: int = 10,
               sweeps_therm: int = 2000, sweeps_measure: int = 10000, measure_interval: int = 1,
               or_per_metropolis: int = 0, step: float = 0.6, adapt_target: float = 0.5, adapt_interval: int = 50,
               renorm_interval: int = 1000, nbins: int = 32, init=None, seed: Optional[int] = None,
               lanes_per_site: int = 0, mode: int = 0, chunk: int = 2000, kernel: int = 0, proposals: int = 0,
               learned=None, checkpoint: Optional[str] = None, checkpoint_interval: int = 0,
               progress=None) -> PTResult:
    """Parallel tempering on the device (gpu_pt.jl:261-316 semantics; exchanges run on
    the device). `gHs` is one GPUTiledHamiltonian or a list of them: every table set
    gets its own ladder over the same kT values (chains of uneven supercells), and
    results are returned ladder-major. With exchange=False the rungs are independent
    chains at their temperatures (run_mc with one chain per temperature).

    Seeds: a numpy Generator seeded with `seed` draws, in order, the initial spins of
    every slot (uniform on S^2) and then one 64-bit device key per slot. `init` replaces
    the random start: one configuration (n_sites x 3) for every rung, or one direction
    (3 values) for the uniform state of every table set.

    learned=(net, env) registers a learned proposal network (scemc.learned) with the
    batch; proposals=3 then draws every Metropolis proposal from it. The wall time
    of the measurement phase is returned in extra["measure_s"].

    checkpoint / checkpoint_interval: every time at least checkpoint_interval sweeps
    have run since the last write (checked at the end of each `chunk`), and at the
    thermalisation -> measurement boundary, the run is written to `checkpoint`
    (gpu_pt kind of src/checkpoint.jl:388-425: progress, the device state of every
    lane, the measurement accumulators); gpu_resume continues it. progress(phase,
    done) is called after each chunk."""
    if isinstance(gHs, GPUTiledHamiltonian):
        gHs = [gHs]
    kts = resolve_kt(temperature, kT)
    R = len(kts)
    if exchange:
        if R < 2:
            raise ValueError(f"parallel tempering needs a ladder of ≥ 2 temperatures; got {R}")
        d = np.diff(kts)
        if not (np.all(d > 0) or np.all(d < 0)):
            raise ValueError(f"the temperature ladder must be strictly monotone; got {kts}")
        if exchange_interval < 1:
            raise ValueError(f"exchange_interval must be ≥ 1; got {exchange_interval}")
    if sweeps_therm < 0 or sweeps_measure < 1 or not (1 <= measure_interval <= sweeps_measure):
        raise ValueError("bad sweep counts / measure_interval")
    if or_per_metropolis < 0 or step <= 0 or not (0 < adapt_target < 1) or adapt_interval < 1 \
            or renorm_interval < 1 or nbins < 2 or chunk < 1 or checkpoint_interval < 0:
        raise ValueError("bad run parameters")
    if or_per_metropolis > 0 and not any(np.any(g.host.site_has_l1) for g in gHs):
        raise ValueError("or_per_metropolis > 0 needs an l = 1 spin channel somewhere")
    if lanes_per_site and not _ispow2(int(lanes_per_site)):
        raise ValueError(f"lanes_per_site must be a power of two (got {lanes_per_site})")
    if seed is None:
        seed = int(np.random.SeedSequence().entropy) & 0xFFFFFFFFFFFFFFFF
    rng = np.random.default_rng(seed)
    configs = []
    for g in gHs:
        if init is None:
            configs += _random_configs(g.n_sites, R, rng)
        else:
            c = np.asarray(init, np.float64).reshape(-1, 3)
            if c.shape[0] == 1:  # one direction: the uniform state of every table set
                c = np.tile(c / np.linalg.norm(c), (g.n_sites, 1))
            configs += [c.copy() for _ in range(R)]
    seeds = rng.integers(0, 2 ** 64, size=R * len(gHs), dtype=np.uint64)
    batch = GPUBatch(gHs, [R] * len(gHs), configs, seeds, step)
    batch.set_betas(np.tile(1.0 / kts, len(gHs)))
    if learned is not None:
        batch.set_learned(*learned)
    run = dict(kts=np.asarray(kts, np.float64), exchange=bool(exchange), exchange_interval=int(exchange_interval),
               sweeps_therm=int(sweeps_therm), sweeps_measure=int(sweeps_measure),
               measure_interval=int(measure_interval), or_per_metropolis=int(or_per_metropolis), step=float(step),
               adapt_target=float(adapt_target), adapt_interval=int(adapt_interval),
               renorm_interval=int(renorm_interval), nbins=int(nbins), seed=int(seed),
               lanes_per_site=int(lanes_per_site), mode=int(mode), chunk=int(chunk), kernel=int(kernel),
               proposals=int(proposals), checkpoint_interval=int(checkpoint_interval))
    ck = _Checkpointer(checkpoint, int(checkpoint_interval), gHs, run)
    return _drive_pt(gHs, batch, run, "therm", 0, None, 0.0, ck, progress)


CHECKPOINT_VERSION = 1


def _tables_fingerprint(gHs) -> str:
    """SHA-256 over every table set's host arrays (the model fingerprint a resume checks)."""
    import hashlib
    h = hashlib.sha256()
    for g in gHs:
        H = g.host
        for name in ("site_ptr", "site_inst", "site_slot", "site_prog", "site_col", "site_col2", "sprog_ptr",
                     "sent_w", "sent_tgt", "color_ptr", "color_sites", "site_active", "site_has_l1"):
            a = getattr(H, name, None)
            if a is not None:
                h.update(name.encode())
                h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


class _Checkpointer:
    """Periodic writer of gpu_pt checkpoints (ck.since / ck.interval of checkpoint.jl)."""

    def __init__(self, path, interval, gHs, run):
        self.path, self.interval, self.run, self.since = path, interval, run, 0
        self.fingerprint = _tables_fingerprint(gHs) if path else ""
        self.shapes = np.array([[g.n_sites, g.host.n_colors] for g in gHs], np.int64)

    def tick(self, n, *args):
        if not self.path or self.interval <= 0:
            return
        self.since += n
        if self.since >= self.interval:
            self.write(*args)

    def write(self, batch, phase, done, accs, measure_s):
        if not self.path:
            return
        import os
        self.since = 0
        d = {"kind": np.array("gpu_pt"), "version": np.array([CHECKPOINT_VERSION], np.int64),
             "fingerprint": np.array(self.fingerprint), "shapes": self.shapes,
             "progress/phase": np.array(phase), "progress/done": np.array([done], np.int64),
             "measure_s": np.array([measure_s]), "state": batch.save_state()}
        for k, v in self.run.items():
            d["run/" + k] = np.asarray(v)
        if accs is not None:
            for i, acc in enumerate(accs):
                d.update(acc.state(f"lane/{i}/accs/"))
        tmp = f"{self.path}.tmp.{os.getpid()}"
        with open(tmp, "wb") as f:
            np.savez(f, **d)
        os.replace(tmp, self.path)


def _run_common(run) -> dict:
    return dict(or_per_metropolis=run["or_per_metropolis"], exchange=run["exchange"],
                exchange_interval=run["exchange_interval"], renorm_interval=run["renorm_interval"],
                lanes_per_site=run["lanes_per_site"], mode=run["mode"], kernel=run["kernel"],
                proposals=run["proposals"])


def _drive_pt(gHs, batch, run, phase, done, accs, measure_s, ck, progress) -> PTResult:
    """The segment loop of gpu_run_pt from (phase, done) on; accs are the measurement
    accumulators when phase is "measure"."""
    kts = run["kts"]
    R = len(kts)
    common = _run_common(run)
    chunk = run["chunk"]
    if phase == "therm":
        total = run["sweeps_therm"]
        while done < total:
            n = min(chunk, total - done)
            batch.run(n, adapt_interval=run["adapt_interval"], adapt_target=run["adapt_target"], phase_done=done,
                      phase_total=total, **common)
            done += n
            if done < total:
                ck.tick(n, batch, "therm", done, None, 0.0)
            if progress is not None:
                progress("therm", done)
        # thermalisation -> measurement boundary: renormalise, fresh counters (gpu_pt.jl:161-179)
        batch.renormalize()
        batch.reset_counters()
        phase, done = "measure", 0
    planned = run["sweeps_measure"] // run["measure_interval"]
    fresh = accs is None
    if fresh:
        accs = [StandardAccumulators(g.host.n_cell_atoms, planned, run["nbins"]) for g in gHs for _ in range(R)]
        ck.write(batch, "measure", 0, accs, measure_s)
    rec_off = [0]
    for g in gHs:
        rec_off.append(rec_off[-1] + R)
    total = run["sweeps_measure"]
    while done < total:
        n = min(chunk, total - done)
        t0 = time.perf_counter()
        batch.run(n, measure_interval=run["measure_interval"], phase_done=done, phase_total=total, **common)
        done += n
        rec = batch.fetch_measurements()
        for i, acc in enumerate(accs):
            li = np.searchsorted(rec_off, i, side="right") - 1
            A = gHs[li].host.n_cell_atoms
            if len(rec):
                acc.push_records(rec[:, i, : 4 + 3 * A])
        measure_s += time.perf_counter() - t0
        if done < total:
            ck.tick(n, batch, "measure", done, accs, measure_s)
        if progress is not None:
            progress("measure", done)
    st = batch.download()
    points = []
    for i, acc in enumerate(accs):
        li = np.searchsorted(rec_off, i, side="right") - 1
        H = gHs[li].host
        kt = float(kts[i - rec_off[li]])
        cnt = st["counters"][i]
        acc_m = cnt[0] / cnt[1] if cnt[1] else np.nan
        acc_o = cnt[2] / cnt[3] if cnt[3] else np.nan
        points.append(TempResult(kt, kt / KB_EV, acc.finalize(kt, H.n_active), acc_m, acc_o, float(st["steps"][i]),
                                 float(st["max_drift"][i])))
    sw = st["swaps"]
    swaps = []
    for li in range(len(gHs)):
        for r in range(R - 1):
            a, b = sw[rec_off[li] + r]
            swaps.append(b / a if a else np.nan)
    finals = [st["configs"][st["slot_of_rung"][i]] for i in range(len(accs))]
    return PTResult(points, np.asarray(swaps), finals, run["seed"],
                    extra=dict(energies=st["energies"], slot_of_rung=st["slot_of_rung"], batch=batch,
                               measure_s=measure_s))


def gpu_resume(path: str, gHs, *, learned=None, checkpoint: Optional[str] = "", checkpoint_interval=None,
               progress=None) -> PTResult:
    """Continues a gpu_run_pt run from its checkpoint and returns the whole run's
    result, bit-identical to the uninterrupted run (resume of src/checkpoint.jl for the
    gpu_pt kind). The caller passes the same table sets (checked against the stored
    fingerprint) and, for a learned run, the same (net, env). By default the resumed
    run keeps writing to `path` at the stored cadence (checkpoint=None disables it;
    checkpoint_interval overrides the cadence). The measurement wall time in
    extra["measure_s"] adds the time before the interruption."""
    if isinstance(gHs, GPUTiledHamiltonian):
        gHs = [gHs]
    with np.load(path, allow_pickle=False) as f:
        d = {k: f[k] for k in f.files}
    if str(d.get("kind", "")) != "gpu_pt" or int(d["version"][0]) != CHECKPOINT_VERSION:
        raise ValueError(f"{path} is not a gpu_pt checkpoint of version {CHECKPOINT_VERSION}")
    if str(d["fingerprint"]) != _tables_fingerprint(gHs):
        raise ValueError("the table sets differ from the checkpointed run's (model fingerprint mismatch)")
    run = {k[4:]: d[k] for k in d if k.startswith("run/")}
    for k in list(run):
        v = run[k]
        if k == "kts":
            run[k] = np.asarray(v, np.float64)
        elif v.dtype == np.bool_:
            run[k] = bool(v)
        elif np.issubdtype(v.dtype, np.integer):
            run[k] = int(v)
        else:
            run[k] = float(v)
    kts = run["kts"]
    R = len(kts)
    configs = [np.tile([0.0, 0.0, 1.0], (g.n_sites, 1)) for g in gHs for _ in range(R)]
    batch = GPUBatch(gHs, [R] * len(gHs), configs, np.arange(1, R * len(gHs) + 1, dtype=np.uint64), run["step"],
                     energies=np.zeros(R * len(gHs)))
    batch.load_state(d["state"])
    if learned is not None:
        batch.set_learned(*learned)
    phase = str(d["progress/phase"])
    done = int(d["progress/done"][0])
    accs = None
    if phase == "measure":
        planned = run["sweeps_measure"] // run["measure_interval"]
        accs = [StandardAccumulators(g.host.n_cell_atoms, planned, run["nbins"]) for g in gHs for _ in range(R)]
        for i, acc in enumerate(accs):
            acc.load_state(f"lane/{i}/accs/", d)
    interval = int(run.get("checkpoint_interval", 0))
    interval = interval if checkpoint_interval is None else int(checkpoint_interval)
    run["checkpoint_interval"] = interval
    ck = _Checkpointer(path if checkpoint == "" else checkpoint, interval, gHs, run)
    return _drive_pt(gHs, batch, run, phase, done, accs, float(d["measure_s"][0]), ck, progress)
