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
