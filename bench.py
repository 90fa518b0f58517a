#!/usr/bin/env python
"""Spin-updates/s of the B200 colour-class sweep.

Default workload (the large frustrated configuration, --workload fcc): fcc 4-site
cell, n^3 cells (--fcc-n, default 64: 1,048,576 spins); l <= 2 pairs to shell 4
(N(0, 1 meV), +0.5 meV isotropic mean on shell 1), NN triangles N(0, 0.1 meV),
Zeeman 2 muB in 0.5 T || [111]; 32 parallel-tempering rungs with kT geometric in
[0.05, 2.0] meV. One step = one compound sweep (Metropolis + 1 overrelaxation
pass) of all 32 rungs followed by an on-device replica-exchange attempt. The spins
alone (32 x 1 M x 16 B = 512 MiB) exceed L2, so no flush is needed. On one GPU the
line also carries, as a labelled extra object, the learned-vs-plain comparison of
the learned-proposal configuration (see --workload learned; --no-learned skips it).

--workload bcc16 (the second benchmark configuration): bcc,
2 sublattices, 16^3 cells (8192 spins); l = 1 and l = 2 pair products to the 3rd
shell (shell means -1.0/-0.3/-0.1 meV, sigma 0.1 meV per (l m, l' m') entry),
l = 1 body-4 plaquettes N(0, 0.05 meV), Zeeman 2 muB in 1 T || z; 5 temperatures
uniform in [0.2, 2.0] meV; colour-class Metropolis + 1 overrelaxation pass per
sweep, FP32 dE with FP64 running energies; seed 2. One step = one compound sweep
(1 Metropolis + 1 overrelaxation pass) of all 5 chains. The working set (~16 MB)
fits in L2, so L2 is flushed (a 256 MiB write) before every timed step.

The metric counts attempts on active sites (Metropolis + overrelaxation) per
second, summed over chains and GPUs. Synthetic, seeded inputs (no fitted model).

--workload pt (the batched parallel-tempering configuration): 4 ladders of 16 rungs
(kT geometric in [0.1, 3.0] meV) on bcc 8^3, 12^3, 16^3 and 24^3 (645,120 spins
per rung set), J1/J2 isotropic l = 1 + (NN, NN, NNN) triangles N(0, 0.1 meV), all
64 chains in one batch. One step = one Metropolis sweep of every chain followed by
an on-device exchange attempt in every ladder.

--workload learned (the learned-proposal configuration): bcc 32^3 (65,536 spins),
J1 = -1.0 / J2 = -0.2 meV isotropic l = 1 plus l = 1 body-4 plaquettes N(0, 0.05 meV),
16 chains at kT geometric in [0.2, 2.0] meV. The network is trained on 200k site
environments from plain-Metropolis chains at the 16 kT values; then the plain
(adaptive-step) and the learned (Metropolis-Hastings) samplers each run 2000
thermalisation and --steps measurement sweeps (default 30000) of the 16 chains,
both started ordered along the model's easy axis (the direction whose uniform state
has the lowest energy; the random plaquette terms make z a hard direction). The
metric is tau_int-corrected independent samples per second, ESS/s = sum over
chains of n_meas / (1 + 2 max(tau_int(E), tau_int(|m|))) over the measurement wall
time; the line reports the learned value with the plain one and their ratio.

--workload l2body3 (not one of the five benchmark configurations): bcc 16^3 with l <= 2
pairs to shell 2 and (NN, NN, NNN) triangles with every member l in {1, 2} (the
body-3-heavy regime of the reference's fitted models), 5 chains, Metropolis + OR; L2
flushed before every step. Compare the default (merged dense body-3 records) with
--kernel 1 (the generic walk of the reference's sparse programs).

--workload fcc_learned (the large frustrated configuration as specified): the fcc
workload with the learned proposal in field mode: the network reads each site's eight
leave-one-out coefficients and kT (the couplings reach the fourth shell, beyond any
raw-spin environment). It is trained on 200k sites from plain chains at the 32 kT
values; then Metropolis
+ OR + exchange and learned Metropolis-Hastings + OR + exchange each run 1000
thermalisation and --steps (default 4000) measured compound sweeps of the 32 rungs.
The metric is tau_int-corrected samples/s, as for --workload learned.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl scemc|reference]
                  [--workload fcc|bcc16|pt|learned|fcc_learned|l2body3]

--impl reference times the FP64 CPU restatement of the reference's
metropolis_sweep!/overrelaxation_sweep! (oracle/, colour-parallel over all host
threads like sweep_tasks) on the same workload; under torchrun only rank 0 runs it.
That arm builds its tables with the oracle alone: libscemc_cuda.so is never loaded.

Roofline convention: B = 16 + 16 + 16 d + 4 A + 4 bytes per attempt (own spin read +
write, d neighbour float4 gathers, one 4-byte word per adjacency entry, site_ptr).
The headline uses A = the merged records per site the kernel walks (one per
distinct pair neighbour, triplet, quad and the body-1 vector; the benchmark
description's count of adjacency entries); the line also gives the fraction with
A = the reference CSR's entries, where the synthetic fcc model writes each bond as
four (l1, l2) templates.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import shutil
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "bcc16": "bcc16_l2_plaquette_zeeman_5T_metropolis+OR",
    "fcc": "fcc{n}_l2_tri_zeeman_32rungs_metropolis+OR+exchange",
    "learned": "bcc32_J1J2_body4_16T_learned_vs_plain",
    "pt": "bcc8-12-16-24_J1J2_triangles_4x16rungs_PT",
    "fcc_learned": "fcc{n}_l2_tri_zeeman_32rungs_learned+OR+exchange_vs_metropolis+OR+exchange",
    "l2body3": "bcc16_l2_pairs_l2_triangles_5T_metropolis+OR",
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def l2_read_gbs(mib: int = 48, reps: int = 40) -> float:
    """Measured L2 read bandwidth (GB/s): the library's probe reads a `mib` MiB buffer,
    which stays in the 126 MB L2, `reps` times in one launch (CUDA events)."""
    import ctypes as C
    from scemc import _lib
    g = C.c_double()
    _lib.check(_lib.lib().scemc_l2_probe(int(mib) << 20, int(reps), C.byref(g)))
    return g.value


def workload(args):
    """(workload name, Workload, exchange after every sweep): the term lists and
    supercells only; no table is built (the reference arm builds its own)."""
    from scemc import models
    if args.workload == "fcc":
        w = models.config5_fcc(n=args.fcc_n, replicas=32)
        return WORKLOADS["fcc"].format(n=args.fcc_n), w, True
    if args.workload == "pt":
        return WORKLOADS["pt"], models.config3_bcc_pt(), True
    if args.workload == "l2body3":
        return WORKLOADS["l2body3"], models.bcc_l2_body3(16), False
    return WORKLOADS["bcc16"], models.config2_bcc_l2(16), False


def library_mapped() -> bool:
    """Whether this process has mapped libscemc_cuda.so."""
    try:
        return "libscemc_cuda.so" in pathlib.Path("/proc/self/maps").read_text()
    except OSError:
        return False


def dram_traffic(workload_name: str, kernel: int):
    """Measured DRAM bytes per attempt of the dominant kernel of the launch form
    (kernel id) on this workload (an ncu capture summarised in
    profiles/dram_traffic.json), or None."""
    p = ROOT / "profiles" / "dram_traffic.json"
    if not p.exists():
        return None
    return json.loads(p.read_text()).get(workload_name, {}).get(str(kernel))


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def learned_comparison(measure: int, therm: int, epochs: int, kernel: int = 0) -> dict:
    """The learned-vs-plain tau_int-corrected samples/s on the bcc 32^3 body-4 model:
    training-set collection, training on the device, then both samplers from the
    ordered state along the easy axis."""
    import torch
    import scemc
    from scemc import learned, models
    n = 32
    w = models.config4_bcc_body4(n)
    H = w.hamiltonians()[0]
    gH = scemc.GPUTiledHamiltonian(H)
    # the random plaquette terms give the ordered phase an easy axis n*; z is a hard
    # direction, and a chain started along z spends its run rotating its whole
    # magnetisation (slowly, with local moves), so both samplers start along n*
    n_star = learned.easy_axis(scemc.GPUTiledHamiltonian(scemc.TiledHamiltonian(2, w.terms, dims=(4, 4, 4))))
    init = np.tile(n_star, (H.n_sites, 1))
    env = learned.environment_table(models.BCC.positions, (n, n, n))
    t0 = time.perf_counter()
    X, Y = learned.collect_training_set(gH, env, w.kts, 200_000, sweeps_therm=2000, snapshots=4, spacing=50, seed=4,
                                        init=init)
    t1 = time.perf_counter()
    net = learned.ProposalNet(seed=4)
    losses = net.train(X, Y, batch=1024, epochs=epochs, lr=1e-3, seed=4)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    kw = dict(kT=w.kts, exchange=False, sweeps_therm=therm, sweeps_measure=measure, seed=4, kernel=kernel, init=init)
    plain = scemc.gpu_run_pt(gH, **kw)
    torch.cuda.nvtx.range_push("timed_steps")  # the learned arm, for a profiler's launch list
    lrn = scemc.gpu_run_pt(gH, learned=(net, env), proposals=3, **kw)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ess_p, _, tau_p = learned.ess_per_second(plain)
    ess_l, _, tau_l = learned.ess_per_second(lrn)
    e_p = np.array([float(p.stats["energy"].mean[0]) for p in plain.points])
    e_l = np.array([float(p.stats["energy"].mean[0]) for p in lrn.points])
    s_p = np.array([float(p.stats["energy"].err[0]) for p in plain.points])
    s_l = np.array([float(p.stats["energy"].err[0]) for p in lrn.points])
    z = np.abs(e_l - e_p) / np.hypot(s_p, s_l)
    return dict(
        workload=WORKLOADS["learned"], metric="tau_int-corrected samples/s", unit="samples/s",
        learned_ess_per_s=ess_l, plain_ess_per_s=ess_p, learned_over_plain=ess_l / ess_p,
        learned_ms_per_sweep=1e3 * lrn.extra["measure_s"] / measure,
        plain_ms_per_sweep=1e3 * plain.extra["measure_s"] / measure, measure_sweeps=measure, therm_sweeps=therm,
        sites_per_chain=H.n_sites, chains=len(w.kts), start="ordered along the easy axis " +
        np.array2string(n_star, precision=4), tau_max_plain=tau_p.tolist(), tau_max_learned=tau_l.tolist(),
        acceptance_plain=[p.acceptance_metropolis for p in plain.points],
        acceptance_learned=[p.acceptance_metropolis for p in lrn.points],
        energy_plain=e_p.tolist(), energy_learned=e_l.tolist(), energy_err_plain=s_p.tolist(),
        energy_err_learned=s_l.tolist(), energy_z=z.tolist(), energy_z_max=float(z.max()),
        training_rows=int(X.shape[0]), epochs=epochs, collect_s=t1 - t0, train_s=t2 - t1,
        train_loss_first_last=[float(losses[0]), float(losses[-1])], _plain=plain, _learned=lrn)


def run_fcc_learned(args) -> int:
    """The large frustrated configuration as specified: learned proposal +
    overrelaxation + replica exchange on fcc n^3 x 32 rungs, against Metropolis +
    overrelaxation + exchange; tau_int-corrected samples/s of both."""
    import torch
    import scemc
    from scemc import learned, models
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.fcc_n
    w = models.config5_fcc(n=n, replicas=32)
    H = w.hamiltonians()[0]
    gH = scemc.GPUTiledHamiltonian(H)
    # field mode: the network reads each site's leave-one-out coefficients (8 numbers for
    # lmax 2) and kT; the model's couplings reach the fourth shell (54 neighbours), which
    # an environment of raw neighbour spins (at most 21 sites) cannot cover
    t0 = time.perf_counter()
    X, Y = learned.collect_field_training_set(gH, w.kts, 200_000, sweeps_therm=1000, snapshots=4, spacing=50,
                                              seed=5, or_per_metropolis=1)
    t1 = time.perf_counter()
    net = learned.ProposalNet(seed=5, field_rows=8)
    losses = net.train(X, Y, batch=1024, epochs=args.epochs, lr=1e-3, seed=5)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    relax = fcc_relaxation(gH, w.kts, net, sweeps=1500, every=25)
    measure = args.steps
    kw = dict(kT=w.kts, exchange=True, exchange_interval=1, or_per_metropolis=1, sweeps_therm=args.therm,
              sweeps_measure=measure, seed=5, kernel=3)
    plain = scemc.gpu_run_pt(gH, **kw)
    lrn = scemc.gpu_run_pt(gH, learned=(net, None), proposals=3, **kw)
    torch.cuda.synchronize()
    ess_p, _, tau_p = learned.ess_per_second(plain)
    ess_l, _, tau_l = learned.ess_per_second(lrn)

    def col(r, name):
        return [float(p.stats[name].mean[0]) for p in r.points], [float(p.stats[name].err[0]) for p in r.points]

    (e_p, s_p), (e_l, s_l) = col(plain, "energy"), col(lrn, "energy")
    z = np.abs(np.subtract(e_l, e_p)) / np.hypot(s_p, s_l)
    line = {"metric": "tau_int-corrected samples/s", "value": ess_l, "unit": "samples/s", "n_gpus": 1,
            "steps": measure, "warmup": args.therm, "ms_per_step": 1e3 * lrn.extra["measure_s"] / measure,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 dE, bf16 network",
            "data": "synthetic",
            "config": {"workload": WORKLOADS["fcc_learned"].format(n=n), "sites_per_chain": H.n_sites,
                       "rungs": len(w.kts), "step": "one compound sweep of every rung (learned Metropolis-Hastings "
                       "or Metropolis, then 1 overrelaxation pass) and an exchange attempt",
                       "plain_ess_per_s": ess_p, "learned_over_plain": ess_l / ess_p,
                       "plain_ms_per_step": 1e3 * plain.extra["measure_s"] / measure,
                       "tau_max_plain": tau_p.tolist(), "tau_max_learned": tau_l.tolist(),
                       "acceptance_plain": [p.acceptance_metropolis for p in plain.points],
                       "acceptance_learned": [p.acceptance_metropolis for p in lrn.points],
                       "swap_acceptance_plain": plain.swap_acceptance.tolist(),
                       "swap_acceptance_learned": lrn.swap_acceptance.tolist(),
                       "energy_plain": e_p, "energy_learned": e_l, "energy_err_plain": s_p,
                       "energy_err_learned": s_l, "energy_z": z.tolist(), "energy_z_max": float(np.max(z)),
                       "training_rows": int(X.shape[0]), "epochs": args.epochs, "collect_s": t1 - t0,
                       "train_s": t2 - t1, "train_loss_first_last": [float(losses[0]), float(losses[-1])],
                       "relaxation": relax}}
    print(json.dumps(line))
    return 0


def fcc_relaxation(gH, kts, net, *, sweeps: int, every: int, seed: int = 11) -> dict:
    """Relaxation from one random start: both arms (Metropolis + OR + exchange, and
    learned Metropolis-Hastings + OR + exchange) run `sweeps` compound sweeps from the
    same random configurations with the same keys, recording every rung's energy each
    `every` sweeps (step adaptation on, as in a thermalisation phase). Per rung, the
    target is the plain arm's final energy (mean of its last four records); the
    learned arm's time to reach it (first record at or below, its sweeps x its seconds
    per sweep) against the plain arm's whole run gives the speed-up in reaching that
    energy."""
    import scemc
    from scemc import models
    R = len(kts)
    n = gH.n_sites
    cfgs = [models.random_config(n, seed + r) for r in range(R)]
    out = {"sweeps": [every * (k + 1) for k in range(sweeps // every)]}
    per_sweep, traces, drift = {}, {}, {}
    for arm in ("plain", "learned"):
        b = scemc.GPUBatch([gH], [R], cfgs, [seed * 100 + r for r in range(R)], 0.6)
        b.set_betas(1.0 / np.asarray(kts))
        if arm == "learned":
            b.set_learned(net, None)
        kw = dict(or_per_metropolis=1, exchange=True, exchange_interval=1, kernel=3, measure_interval=every,
                  phase_total=sweeps, proposals=3 if arm == "learned" else 0, adapt_interval=50, adapt_target=0.5)
        t0 = time.perf_counter()
        b.run(sweeps, **kw)
        per_sweep[arm] = (time.perf_counter() - t0) / sweeps
        rec = b.fetch_measurements()  # (records, rungs, columns); column 0 the energy (eV)
        traces[arm] = rec[:, :R, 0] / n
        # the running energies (FP32 dE, fixed-point sums) against the FP64 recompute
        run_e = b.download()["energies"]
        drift[arm] = max(abs(run_e[k] - b.total_energy(k)) / n for k in range(R))
        del b
    target = traces["plain"][-4:].mean(axis=0)
    speedups, reach = [], []
    for r in range(R):
        hit = np.nonzero(traces["learned"][:, r] <= target[r])[0]
        k = int(hit[0]) + 1 if len(hit) else None
        reach.append(None if k is None else every * k)
        speedups.append(None if k is None else (sweeps * per_sweep["plain"]) / (every * k * per_sweep["learned"]))
    got = [x for x in speedups if x is not None]
    out.update({"plain_s_per_sweep": per_sweep["plain"], "learned_s_per_sweep": per_sweep["learned"],
                "max_drift_eV_per_site": drift,
                "plain_energy_ueV_per_site": (1e6 * traces["plain"].mean(axis=1)).tolist(),
                "learned_energy_ueV_per_site": (1e6 * traces["learned"].mean(axis=1)).tolist(),
                "learned_sweeps_to_plain_final": reach, "speedup_to_plain_final": speedups,
                "speedup_median": float(np.median(got)) if len(got) == R else None,
                "speedup_min": float(np.min(got)) if len(got) == R else None})
    return out


def run_learned(args) -> int:
    """The learned-vs-plain tau_int-corrected samples/s on the bcc 32^3 body-4 model."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    measure = args.steps
    c = learned_comparison(measure, args.therm, args.epochs, args.kernel)
    plain, lrn = c.pop("_plain"), c.pop("_learned")
    ess_l, ess_p = c["learned_ess_per_s"], c["plain_ess_per_s"]
    ms = c["learned_ms_per_sweep"]
    line = {"metric": "tau_int-corrected samples/s", "value": ess_l, "unit": "samples/s", "n_gpus": 1,
            "steps": measure, "warmup": args.therm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 dE, bf16 network", "data": "synthetic",
            "config": dict(c, step="one sweep of every chain (Metropolis or learned Metropolis-Hastings)",
                           kernel=args.kernel or "auto")}
    print(json.dumps(line))
    return 0


def run_cpu_reference(w, steps: int, warmup: int, budget_s: float, max_chains: int = 0):
    """Times the oracle's compound sweep (Metropolis + 1 OR) of the workload's chains
    on the first supercell (the first max_chains of them when > 0, a bounded sample of
    a large batch) on all host threads; the tables are the oracle's own. Returns
    (attempts/s, threads, sample description, per-step ms, sites per chain)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    from scemc import models
    dims = tuple(w.dims_list[0])
    OH = O.OracleHamiltonian(w.n_cell_atoms, w.terms, dims, magmoms=w.magmoms, field=w.field)
    n_sites = w.n_cell_atoms * int(np.prod(dims))
    threads = max(1, os.cpu_count() or 1)
    kts = w.kts[:max_chains] if max_chains > 0 else w.kts
    chains = [O.OracleChain(OH, models.random_config(n_sites, 100 + i), seed=1000 + i) for i in range(len(kts))]

    def step():
        att = 0
        for ch, kt in zip(chains, kts):
            c0 = ch.get()[3]
            ch.sweeps(1.0 / kt, 1, n_or=w.or_per_metropolis, threads=threads)
            c1 = ch.get()[3]
            att += int((c1[1] - c0[1]) + (c1[3] - c0[3]))
        return att

    for _ in range(warmup):
        step()
    tot_att, tot_t, n = 0, 0.0, 0
    for _ in range(steps):
        t0 = time.perf_counter()
        tot_att += step()
        tot_t += time.perf_counter() - t0
        n += 1
        if tot_t > budget_s:
            break
    sample = (f"{n} compound sweeps (Metropolis + {w.or_per_metropolis} OR) of {len(kts)} of {len(w.kts)} chains x "
              f"{n_sites} spins, FP64 oracle, {threads} threads, {cpu_model()}")
    return tot_att / tot_t, threads, sample, 1e3 * tot_t / n, n_sites


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # raw samples beside the bench's other outputs (SCEMC_BENCH_OUT, default ./bench_out)
        out = pathlib.Path(os.environ.get("SCEMC_BENCH_OUT", ROOT / "bench_out"))
        self.path = out / f"clocks_rank{index}.csv"

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.path.parent.mkdir(parents=True, exist_ok=True)
        self.fh = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.fh,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 100 fcc, 2000 bcc16)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="scemc", choices=["scemc", "reference"])
    ap.add_argument("--workload", default="fcc", choices=sorted(WORKLOADS))
    ap.add_argument("--no-learned", action="store_true",
                    help="fcc on one GPU: skip the learned-vs-plain extra object")
    ap.add_argument("--fcc-n", type=int, default=64, help="cells per edge of the fcc workload")
    ap.add_argument("--mode", type=int, default=0, help="0 auto, 1 per-colour launches, 2 persistent, 3 graph")
    ap.add_argument("--kernel", type=int, default=0,
                    help="0 auto, 1 generic, 2 row-parallel, 3 replica-parallel, 4 chain-resident cluster, "
                         "5 replica-parallel with tensor-core pair records")
    ap.add_argument("--lanes", type=int, default=0, help="lanes per site (0 = autotuned)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--therm", type=int, default=2000,
                    help="learned workloads: thermalisation sweeps per arm (fcc_learned: 1000)")
    ap.add_argument("--epochs", type=int, default=20, help="learned workload: training epochs")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    big = args.workload in ("fcc", "pt")
    if args.steps is None:
        # learned: plain Metropolis's tau_int is 100-200 sweeps here, so its log-binning
        # estimate needs a few 10^4 sweeps (10^4 underestimates it by a third)
        args.steps = {"fcc": 100, "learned": 30000, "pt": 200, "fcc_learned": 4000}.get(args.workload, 2000)
    if args.workload == "fcc_learned":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned proposal; "
                              "its plain sampler is the plain arm inside this workload's line"}))
            return 0
        if args.therm == 2000:
            args.therm = 1000
        return run_fcc_learned(args)
    if args.workload == "learned":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned proposal; "
                              "its plain sampler is the plain arm inside this workload's line"}))
            return 0
        return run_learned(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        name, w, _ = workload(args)
        steps = max(1, min(args.steps, 50))
        v, threads, sample, ms, n_sites = run_cpu_reference(w, steps, min(args.warmup, 3) if not big else 1,
                                                            args.cpu_budget, max_chains=1 if big else 0)
        line = {"metric": "spin-updates/s", "value": v, "unit": "attempts/s", "n_gpus": args.gpus,
                "steps": steps, "warmup": min(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": name, "sites_per_chain": n_sites, "chains": len(w.kts),
                           "libscemc_cuda_loaded": library_mapped()},
                "impl": "reference",
                "cpu_baseline": {"value": v, "unit": "attempts/s", "cores": threads, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": v, "unit": "attempts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    import scemc
    from scemc import ranks

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_
        dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_

    name, w, exchange = workload(args)
    Hs = w.hamiltonians()
    gHs = [scemc.GPUTiledHamiltonian(h) for h in Hs]
    st_ = [g.stats() for g in gHs]
    wts = np.array([h.n_sites for h in Hs], float)
    d_mean = float(np.dot([x[0] for x in st_], wts) / wts.sum())
    a_mean = float(np.dot([x[1] for x in st_], wts) / wts.sum())
    r_mean = float(np.dot([g.records_per_site() for g in gHs], wts) / wts.sum())
    table_bytes = int(sum(x[2] for x in st_))
    R = len(w.kts)
    rng = np.random.default_rng(2 + 1000 * rank)
    configs = [models_random(h.n_sites, rng) for h in Hs for _ in range(R)]
    seeds = ranks.rank_keys(2, rank, R * len(Hs))
    batch = scemc.GPUBatch(gHs, [R] * len(Hs), configs, seeds, 0.6)
    batch.set_betas(np.tile(1.0 / w.kts, len(Hs)))
    H = Hs[0]
    n_or = w.or_per_metropolis
    form = dict(lanes_per_site=args.lanes, mode=args.mode, kernel=args.kernel)
    # exchange after every sweep: phase_total far ahead so that no sweep is a phase's last
    xkw = dict(exchange=True, exchange_interval=1, phase_total=1 << 62) if exchange else {}
    p = scemc.GPUBatch.params(1, or_per_metropolis=n_or, **form, **xkw)
    stream = torch.cuda.ExternalStream(batch.stream())
    # the fcc spins alone (512 MiB) exceed L2; the other workloads' spins and tables fit, so
    # L2 is flushed before every timed step
    flush_l2 = args.workload != "fcc"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if flush_l2 else None

    def one_step():
        batch.run_async(p)
        batch.sync()

    tuned = None
    if args.mode == 0 and args.lanes == 0 and args.kernel == 0:  # pick the launch form by timing them
        tuned = batch.autotune(or_per_metropolis=n_or, sweeps_per_trial=2 if big else 10)
    # thermalise a little so acceptance rates are representative, then warm up
    batch.run(10 if big else 200, or_per_metropolis=n_or, **form)
    for _ in range(args.warmup):
        one_step()

    cnt0 = batch.download()["counters"].copy()
    launches0 = batch.launches()
    clocks = ClockSampler(local)
    batch.profile(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms = []
    torch.cuda.nvtx.range_push("timed_steps")  # lets a profiler select the timed launches
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            if flush is not None:
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        batch.run_async(p)
        e1.record(stream)
        batch.sync()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    kern_ms, passes = batch.kernel_time()
    batch.profile(False)
    st1 = batch.download()
    cnt1 = st1["counters"]
    launches = batch.launches() - launches0
    att = cnt1 - cnt0
    attempts = int(att[:, 1].sum() + att[:, 3].sum())
    total_ms = float(np.sum(step_ms))
    total_ms_max, attempts_all = ranks.aggregate(total_ms, attempts, dist, device="cuda")
    value = attempts_all / (total_ms_max * 1e-3)

    # roofline of the sweep kernel: algorithmic bytes per attempt (own spin read +
    # write, d neighbour float4 gathers, one 4-byte word per adjacency entry, site_ptr).
    # Headline: the adjacency entries are the merged records the kernel walks (one per
    # distinct pair neighbour, triplet, quad and body-1 vector); beside it, the same
    # with the reference CSR's entries (the fcc model writes each bond as four (l1, l2)
    # templates, so its CSR has about three times as many).
    A_kernel = r_mean if r_mean > 0 else a_mean
    B = 16 + 16 + 16 * d_mean + 4 * A_kernel + 4
    B_ref = 16 + 16 + 16 * d_mean + 4 * a_mean + 4
    hbm, peak_kind = peaks()
    achieved = attempts * B / (kern_ms * 1e-3) / 1e9 if kern_ms > 0 else None
    achieved_ref = attempts * B_ref / (kern_ms * 1e-3) / 1e9 if kern_ms > 0 else None
    run_kernel = args.kernel or (tuned or {}).get("kernel") or 0
    tr = dram_traffic(name, run_kernel)
    traffic = tr["bytes_per_attempt"] * attempts / max(passes, 1) if tr else None
    # the bcc16 and PT working sets (spins and tables) fit in L2: their sweeps are judged
    # against the measured L2 bandwidth (and are latency-bound well below it)
    l2 = l2_read_gbs()
    bound, peak = ("hbm", hbm) if not flush_l2 else ("l2", l2)

    # end-to-end through the C ABI with host buffers in pinned memory: upload every
    # chain's FP64 spins and energy, one step (compound sweep, plus the exchange where
    # the workload has one), download the full state into the same host buffer
    pinned = scemc.PinnedHost(3 * batch.n_sites_total)
    host_cfg = pinned.array
    host_cfg[:] = np.concatenate([c.reshape(-1) for c in st1["configs"]])
    host_en = st1["energies"].copy()
    e2e_steps = 3 if big else max(10, min(args.steps, 100))
    e2e_kw = dict(or_per_metropolis=n_or, **form, **xkw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d2h = 0
    for _ in range(e2e_steps):
        batch.upload(host_cfg, host_en)
        batch.run(1, **e2e_kw)
        st = batch.download(out=host_cfg)
        host_en = st["energies"]
        d2h = sum(np.asarray(v).nbytes for k, v in st.items() if k != "configs") + host_cfg.nbytes
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    pinned.close()
    per_step_att = attempts / args.steps
    e2e_value = per_step_att * e2e_steps * world / e2e_s
    h2d = host_cfg.nbytes + host_en.nbytes

    cpu = None
    if rank == 0 and world == 1:
        v, threads, sample, _, _ = run_cpu_reference(w, 50, 1, args.cpu_budget, max_chains=1 if big else 0)
        cpu = {"value": v, "unit": "attempts/s", "cores": threads, "kind": "port", "sample": sample}
    extra = None
    if rank == 0 and world == 1 and args.workload == "fcc" and not args.no_learned:
        del batch, pinned
        extra = learned_comparison(30000, 2000, 20)
        extra.pop("_plain"), extra.pop("_learned")

    if rank == 0:
        line = {
            "metric": "spin-updates/s", "value": value, "unit": "attempts/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": name, "sites_per_chain": [h.n_sites for h in Hs] if len(Hs) > 1 else H.n_sites,
                       "chains_per_gpu": R * len(Hs),
                       "compound_sweep": f"1 Metropolis + {n_or} OR" + (" + exchange" if exchange else ""),
                       "l2": ("inputs larger than L2 (spins alone %.0f MiB)" % (R * wts.sum() * 16 / 2 ** 20))
                       if not flush_l2
                       else "flushed (256 MiB) before every step",
                       "lanes_per_site": args.lanes or "auto", "mode": args.mode or "auto",
                       "kernel": args.kernel or "auto", "autotuned": tuned,
                       "d_mean": d_mean, "A_mean": a_mean, "table_bytes": table_bytes,
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": bound, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "kernel": tr.get("kernel") if tr else None,
                         "limiter": "latency: serial colour steps of a dependent record walk, far below the "
                                    "L2 and HBM rooflines" if bound == "l2" else
                         "issue and latency (operand splits, neighbour gathers, the per-replica triangle "
                         "walk); tensor pipe and HBM below their peaks" if run_kernel == 5 else
                         "L1 data path and issue (the neighbour gathers and coupling blocks); HBM "
                         "below its peak",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "peak_kind": peak_kind if bound == "hbm" else "measured L2 read (this run)",
                         "hbm_peak": hbm, "frac_of_hbm": (achieved / hbm) if achieved else None,
                         "l2_read_gbs": l2, "bytes_per_attempt": B,
                         "adjacency_entries": "kernel records (%.1f per site)" % A_kernel,
                         "achieved_reference_csr": achieved_ref,
                         "frac_reference_csr": (achieved_ref / hbm) if achieved_ref else None,
                         "bytes_per_attempt_reference_csr": B_ref,
                         "traffic_source": tr.get("source") if tr else None,
                         "kernel_ms_per_pass": kern_ms / max(passes, 1), "passes": passes},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "attempts/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if extra is not None:
            line["learned_vs_plain"] = extra
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def models_random(n, rng):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


if __name__ == "__main__":
    sys.exit(main())
