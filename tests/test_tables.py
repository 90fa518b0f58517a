"""The package's table builder against the oracle's (two independent restatements of
src/hamiltonian.jl), the synthetic workloads' shapes, the host statistics, and the
C-ABI library's exported surface. CPU only."""
import ctypes as C
import pathlib
import re

import numpy as np
import pytest

import oracle as O
import scemc
from scemc import _lib, models

ROOT = pathlib.Path(__file__).resolve().parents[1]

ARRAYS = ["inst_term", "inst_ptr", "inst_sites", "site_ptr", "site_inst", "site_slot", "site_prog", "sprog_ptr",
          "sent_w", "sent_tgt", "sfac_ptr", "sfac_row", "sfac_slot", "site_col", "site_col2", "pent_row",
          "pent_row2", "eprog_ptr", "eent_w", "efac_ptr", "efac_row", "term_coef", "color_ptr", "color_sites",
          "site_has_l1", "site_active"]

ZB = (0.3, -1.2, 2.0)

FIXTURES = [
    ("dimer", 4, models.dimer_terms(), (1, 1, 1), {}),
    ("dimer zeeman", 4, models.dimer_terms(), (2, 1, 1), dict(magmoms=[2.2, 2.2, 1.0, 0.0], field=ZB)),
    ("biquadratic", 2, models.biquadratic_terms(3), (2, 2, 2), {}),
    ("biquadratic zeeman", 2, models.biquadratic_terms(3), (2, 2, 2), dict(magmoms=[1.5, 0.7], field=ZB)),
    ("zeeman only", 2, [], (2, 2, 1), dict(magmoms=[1.0, 2.0], field=ZB)),
    ("chain", 1, models.chain_terms(-0.05), (4, 4, 2), {}),
    ("threebody", 1, models.threebody_terms(0.05), (4, 2, 2), {}),
    ("fourbody", 1, models.fourbody_terms(0.03), (4, 2, 2), {}),
    ("mixed", 2, models.mixed_terms(7), (2, 2, 1), {}),
    ("high l", 1, models.highl_terms(11, 4), (3, 2, 1), {}),
    ("sc J1J2", 1, models.config1_sc().terms, (4, 4, 4), {}),
    ("bcc l2 plaq zeeman", 2, models.config2_bcc_l2().terms, (3, 3, 3), dict(magmoms=[2.0, 2.0], field=[0, 0, 1.0])),
    ("bcc triangles", 2, models.config3_bcc_pt().terms, (3, 3, 3), {}),
    ("bcc body4", 2, models.config4_bcc_body4().terms, (3, 3, 3), {}),
    ("fcc l2 tri", 4, models.config5_fcc(n=2).terms, (3, 3, 3), dict(magmoms=[2.0] * 4, field=[0.3, 0.3, 0.3])),
    ("bcc l2 body3", 2, models.bcc_l2_body3(3).terms, (3, 3, 3), {}),
]


@pytest.mark.parametrize("name,nca,terms,dims,kw", FIXTURES, ids=[f[0] for f in FIXTURES])
def test_builder_matches_oracle(name, nca, terms, dims, kw):
    H = scemc.TiledHamiltonian(nca, terms, dims=dims, **kw)
    OH = O.OracleHamiltonian(nca, terms, dims, **kw)
    for k in ("n_sites", "nlm", "lmax", "n_colors", "n_active"):
        assert getattr(H, k) == getattr(OH, k), k
    arrs = H.arrays()
    for name_ in ARRAYS:
        a, b = np.asarray(arrs[name_]), OH.array(name_)
        assert a.shape == b.shape, name_
        if a.dtype.kind == "f":
            np.testing.assert_array_equal(a, b, err_msg=name_)
        else:
            np.testing.assert_array_equal(a.astype(np.int64), b.astype(np.int64), err_msg=name_)


def test_builder_errors():
    with pytest.raises(ValueError):
        scemc.TiledHamiltonian(1, [])
    with pytest.raises(ValueError):
        scemc.TiledHamiltonian(1, models.chain_terms(0.05), dims=(1, 1, 1))  # member sites fold together
    with pytest.raises(ValueError):
        scemc.TiledHamiltonian(1, models.dimer_terms())  # atom 2 outside 1:1
    bad = models.chain_terms(0.05)
    bad[0].shifts = [(1, 0, 0), (2, 0, 0)]
    with pytest.raises(ValueError):
        scemc.TiledHamiltonian(1, bad, dims=(4, 1, 1))
    with pytest.raises(ValueError):
        scemc.TiledHamiltonian(1, models.chain_terms(0.05), dims=(4, 1, 1), field=(0, 0, 1))


def test_workload_shapes():
    """Distinct neighbours d and adjacency entries A of the workloads."""
    H1 = models.config1_sc().hamiltonians()[0]
    assert H1.n_sites == 512 and H1.lmax == 1
    assert np.all(np.diff(H1.site_ptr) == 18)
    H2 = models.config2_bcc_l2(n=4).hamiltonians()[0]
    assert H2.n_sites == 128 and H2.lmax == 2
    # 26 neighbours x 4 (l1,l2) blocks + 12 plaquettes + 1 Zeeman
    assert np.all(np.diff(H2.site_ptr) == 26 * 4 + 12 + 1)
    w3 = models.config3_bcc_pt()
    assert [d[0] for d in w3.dims_list] == [8, 12, 16, 24] and len(w3.kts) == 16
    H3 = models.TiledHamiltonian(2, w3.terms, dims=(4, 4, 4))
    assert np.all(np.diff(H3.site_ptr) == 8 + 6 + 36)
    H5 = models.config5_fcc(n=3).hamiltonians()[0]
    assert np.all(np.diff(H5.site_ptr) == 54 * 4 + 24 + 1)


def test_header_symbols_exported():
    """Every entry point declared in include/scemc.h is exported and bound."""
    hdr = (ROOT / "include" / "scemc.h").read_text()
    names = set(re.findall(r"^int32_t (scemc_\w+)\(", hdr, flags=re.M))
    assert len(names) >= 25
    L = C.CDLL(str(_lib.LIB_PATH))
    for n in names:
        assert hasattr(L, n), n
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert names == bound
    assert _lib.lib().scemc_version() >= 100


def test_color_helper_and_error_path():
    H = scemc.TiledHamiltonian(1, models.chain_terms(0.05), dims=(4, 1, 1))
    assert H.n_colors == 2
    L = _lib.lib()
    out = np.zeros(4, np.int32)
    n = C.c_int32()
    rc = L.scemc_color_sites(4, None, None, None, None, None, _lib.ptr(out, C.c_int32), C.byref(n))
    assert rc == _lib.ERR_ARG and "NULL" in _lib.last_error()


def test_stats_jackknife_and_binstore():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(1000)
    s = scemc.stats.BinStore(1, 31, 32)
    s.push_many(x)
    m = s.bin_means()[:, 0]
    assert len(m) == 32
    est, err = scemc.jackknife(lambda a: a, [m])
    assert est == pytest.approx(m.mean()) and err == pytest.approx(m.std(ddof=1) / np.sqrt(32), rel=1e-10)
    with pytest.raises(ValueError):
        scemc.jackknife(lambda a: a, [m[:1]])
