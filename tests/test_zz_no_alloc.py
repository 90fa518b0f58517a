"""The allocation-free energy recompute, checked through the C ABI against the
allocating entry point.

scemc_total_energy_static serves callers that cannot allocate device memory at the
moment they need an energy: a host whose own pool allocator owns all device memory
and only lends the library its buffers, or a time-critical loop that must not pay
cudaMalloc's device-wide synchronisation. It must give the same energies as
scemc_total_energy on the same spins, on every call. This file is collected last
so that a failure here cannot hide the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import scemc
from scemc import _lib, models

pytestmark = pytest.mark.gpu


def test_static_energy_matches_allocating_entry_point(gpu):
    import torch

    w = models.config2_bcc_l2(n=5)
    H = w.hamiltonians()[0]
    gH = scemc.GPUTiledHamiltonian(H)
    R = 3
    cfgs = [models.random_config(H.n_sites, 40 + r) for r in range(R)]
    b = scemc.GPUBatch([gH], [R], cfgs, [1, 2, 3], 0.6)
    ref = np.array([b.total_energy(r) for r in range(R)])
    # caller-owned device buffers holding the same FP32 spins as the batch (which
    # renormalised them on creation), in the library's layout spins[site * R + r]
    dev_cfgs = b.download()["configs"]
    host = np.zeros((H.n_sites, R, 4), np.float32)
    for r, c in enumerate(dev_cfgs):
        host[:, r, :3] = c
    spins = torch.from_numpy(host).cuda()
    out = torch.zeros(R, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    L = _lib.lib()
    for _ in range(2):  # two calls in a row share (and reuse) the fixed scratch
        out.fill_(float("nan"))
        rc = L.scemc_total_energy_static(gH.h, C.c_void_p(spins.data_ptr()), R, C.c_void_p(out.data_ptr()),
                                         C.c_void_p(stream.cuda_stream))
        assert rc == _lib.OK, _lib.last_error()
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=1e-15)
    # a request larger than the fixed scratch is refused with a clear error
    rc = L.scemc_total_energy_static(gH.h, C.c_void_p(spins.data_ptr()), 70000, C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.ERR_ARG and "exceeds the fixed scratch" in _lib.last_error()


def test_static_energy_replica_limit(gpu):
    """One launch-grid row per replica: 65535 replicas are served, 65536 are refused
    with SCEMC_ERR_ARG even where the partial sums would fit the scratch (one chunk
    of instances, the 4-site dimer cell)."""
    import torch

    H = models.dimer()
    gH = scemc.GPUTiledHamiltonian(H)
    OH = O.OracleHamiltonian(4, models.dimer_terms(), (1, 1, 1))
    R = 65535
    rng = np.random.default_rng(5)
    v = rng.standard_normal((H.n_sites, R, 3))
    v /= np.linalg.norm(v, axis=2, keepdims=True)
    host = np.zeros((H.n_sites, R, 4), np.float32)
    host[:, :, :3] = v
    spins = torch.from_numpy(host).cuda()
    out = torch.full((R + 1,), float("nan"), dtype=torch.float64, device="cuda")
    L = _lib.lib()
    rc = L.scemc_total_energy_static(gH.h, C.c_void_p(spins.data_ptr()), R, C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.OK, _lib.last_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for r in (0, 1, R // 2, R - 1):
        E = OH.total_energy(host[:, r, :3].astype(np.float64))
        assert abs(got[r] - E) <= 1e-12 * max(1.0, abs(E)), (r, got[r], E)
    assert np.isnan(got[R])  # nothing beyond the replicas asked for is written
    rc = L.scemc_total_energy_static(gH.h, C.c_void_p(spins.data_ptr()), R + 1, C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.ERR_ARG and "65535" in _lib.last_error()


def test_static_energy_refuses_another_current_device(gpu):
    """The tables' device must be current: on another device the kernels would read
    the tables through pointers of a different GPU."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    H = models.dimer()
    with torch.cuda.device(0):
        gH = scemc.GPUTiledHamiltonian(H)
    with torch.cuda.device(1):
        spins = torch.zeros((H.n_sites, 1, 4), dtype=torch.float32, device="cuda")
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        rc = _lib.lib().scemc_total_energy_static(gH.h, C.c_void_p(spins.data_ptr()), 1,
                                                  C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.ERR_ARG and "make that device current" in _lib.last_error()
