"""Checkpoint and resume of the device PT driver (the gpu_pt kind of
src/checkpoint.jl:388-456): the measurement accumulators' state round trip (CPU),
the batch state blob's guards, and a run interrupted in either phase and resumed
equals the uninterrupted run bit for bit (B200, -m gpu)."""
import numpy as np
import pytest

import scemc
from scemc import _lib, models
from scemc.stats import StandardAccumulators


def test_accumulator_state_round_trip():
    rng = np.random.default_rng(3)
    a = StandardAccumulators(2, planned=200, nbins=8)
    b = StandardAccumulators(2, planned=200, nbins=8)
    first, second = rng.standard_normal((77, 10)), rng.standard_normal((123, 10))
    a.push_records(first)
    b.load_state("x/", a.state("x/"))
    a.push_records(second)
    b.push_records(second)
    fa, fb = a.finalize(0.5, 16), b.finalize(0.5, 16)
    for k in fa:
        for f in ("mean", "err", "tau_int"):
            np.testing.assert_array_equal(getattr(fa[k], f), getattr(fb[k], f))
        assert fa[k].count == fb[k].count
    with pytest.raises(ValueError):
        StandardAccumulators(2, planned=400, nbins=8).load_state("x/", a.state("x/"))


def _same_result(p, q):
    for a, b in zip(p.points, q.points):
        for k in a.stats:
            for f in ("mean", "err", "tau_int"):
                np.testing.assert_array_equal(getattr(a.stats[k], f), getattr(b.stats[k], f), err_msg=k)
        assert (a.acceptance_metropolis, a.final_step, a.max_drift) == \
               (b.acceptance_metropolis, b.final_step, b.max_drift)
        assert a.acceptance_or == b.acceptance_or or (np.isnan(a.acceptance_or) and np.isnan(b.acceptance_or))
    np.testing.assert_array_equal(p.swap_acceptance, q.swap_acceptance)
    for x, y in zip(p.final_configs, q.final_configs):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(p.extra["energies"], q.extra["energies"])


class _Stop(Exception):
    pass


@pytest.mark.gpu
@pytest.mark.parametrize("stop_at,resume_from", [(("therm", 60), ("therm", 40)), (("measure", 60), ("measure", 40))])
def test_interrupted_run_resumes_bit_identically(gpu, tmp_path, stop_at, resume_from):
    w = models.config2_bcc_l2(3)
    H = scemc.TiledHamiltonian(2, w.terms, dims=(3, 3, 3), magmoms=w.magmoms, field=w.field)
    gH = scemc.GPUTiledHamiltonian(H)
    kw = dict(kT=[0.3e-3, 0.6e-3, 1.2e-3, 2.0e-3], sweeps_therm=60, sweeps_measure=120, chunk=20, seed=5,
              exchange_interval=3, or_per_metropolis=1, adapt_interval=10, renorm_interval=30)
    ref = scemc.gpu_run_pt(gH, **kw)
    path = str(tmp_path / "run.ckpt.npz")

    def stop(phase, done):
        if (phase, done) == stop_at:
            raise _Stop

    with pytest.raises(_Stop):
        scemc.gpu_run_pt(gH, checkpoint=path, checkpoint_interval=40, progress=stop, **kw)
    with np.load(path) as f:
        assert (str(f["progress/phase"]), int(f["progress/done"][0])) == resume_from
    seen = []
    res = scemc.gpu_resume(path, gH, progress=lambda ph, d: seen.append((ph, d)))
    assert seen[0] == (resume_from[0], resume_from[1] + 20)
    _same_result(ref, res)
    # another model is refused
    H2 = scemc.TiledHamiltonian(2, models.config4_bcc_body4().terms, dims=(3, 3, 3))
    with pytest.raises(ValueError):
        scemc.gpu_resume(path, scemc.GPUTiledHamiltonian(H2))


@pytest.mark.gpu
def test_state_blob_guards(gpu):
    H = scemc.TiledHamiltonian(1, models.chain_terms(0.05), dims=(8, 1, 1))
    gH = scemc.GPUTiledHamiltonian(H)
    b = scemc.GPUBatch([gH], [3], [models.random_config(8, r) for r in range(3)], [1, 2, 3], 0.5)
    blob = b.save_state()
    other = scemc.GPUBatch([gH], [2], [models.random_config(8, r) for r in range(2)], [1, 2], 0.5)
    with pytest.raises(_lib.ScemcArgumentError):
        other.load_state(blob)
    with pytest.raises(_lib.ScemcArgumentError):
        b.load_state(blob[: blob.size // 2])
    bad = blob.copy()
    bad[0] ^= 0xFF
    with pytest.raises(_lib.ScemcArgumentError):
        b.load_state(bad)
    b.run(5, or_per_metropolis=1)
    after = b.download()
    b.load_state(blob)  # rewinds the chains
    b.run(5, or_per_metropolis=1)
    again = b.download()
    for x, y in zip(after["configs"], again["configs"]):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(after["energies"], again["energies"])
