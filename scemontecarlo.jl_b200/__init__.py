"""B200-native chain-level spin Monte Carlo sweep for SCEMonteCarlo.jl Hamiltonians.

The compute path is libscemc_cuda.so (hand-written sm_100a CUDA behind the C ABI of
include/scemc.h). This package is the host side: the table builder that produces the
reference's flat tiled-Hamiltonian layout, the synthetic workloads, the statistics
of a run, and the reference-named API over the C ABI.
"""
from .hamiltonian import KB_EV, MU_B_EV_T, N1, MultipoleTerm, TiledHamiltonian, resolve_kt
from .gpu import (ChainState, GPUBatch, GPUChainState, GPUTiledHamiltonian, PinnedHost, from_host,
                  gpu_energy_gradient, gpu_metropolis_sweep, gpu_overrelaxation_sweep, gpu_resume, gpu_run_pt,
                  gpu_run_sweeps, swap_payload, to_host)
from .stats import BinStore, LogBinner, ObservableStat, PTResult, TempResult, jackknife
from . import models
from ._lib import ScemcArgumentError, ScemcError

__all__ = [
    "KB_EV", "MU_B_EV_T", "N1", "MultipoleTerm", "TiledHamiltonian", "resolve_kt", "ChainState", "GPUBatch",
    "GPUChainState", "GPUTiledHamiltonian", "PinnedHost", "from_host", "gpu_energy_gradient", "gpu_metropolis_sweep", "gpu_overrelaxation_sweep",
    "gpu_resume", "gpu_run_pt", "gpu_run_sweeps", "swap_payload", "to_host", "BinStore", "LogBinner", "ObservableStat",
    "PTResult", "TempResult", "jackknife", "models", "ScemcArgumentError", "ScemcError",
]
