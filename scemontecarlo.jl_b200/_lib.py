"""ctypes binding of libscemc_cuda.so (the C ABI declared in include/scemc.h).

Loading fails loudly when the library has not been built: there is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libscemc_cuda.so"

OK, ERR_ARG, ERR_UNSUPPORTED, ERR_CUDA, ERR_TIMEOUT, ERR_EXHAUSTED, ERR_NUMERIC = range(7)

I32P = C.POINTER(C.c_int32)
I8P = C.POINTER(C.c_int8)
U8P = C.POINTER(C.c_uint8)
F64P = C.POINTER(C.c_double)
F32P = C.POINTER(C.c_float)
I64P = C.POINTER(C.c_int64)
U64P = C.POINTER(C.c_uint64)


class TablesDesc(C.Structure):
    _fields_ = [
        ("n_sites", C.c_int32), ("nlm", C.c_int32), ("lmax", C.c_int32), ("n_colors", C.c_int32),
        ("n_active", C.c_int32), ("n_cell_atoms", C.c_int32),
        ("n_adj", C.c_int64), ("n_inst", C.c_int64), ("n_inst_sites", C.c_int64), ("n_sprog", C.c_int64),
        ("n_sent", C.c_int64), ("n_sfac", C.c_int64), ("n_terms", C.c_int64), ("n_eent", C.c_int64),
        ("n_efac", C.c_int64),
        ("site_ptr", I32P), ("site_inst", I32P), ("site_slot", I8P), ("inst_term", I32P), ("inst_ptr", I32P),
        ("inst_sites", I32P), ("site_prog", I32P), ("sprog_ptr", I32P), ("sent_w", F64P), ("sent_tgt", I32P),
        ("sfac_ptr", I32P), ("sfac_row", I32P), ("sfac_slot", I8P), ("site_col", I32P), ("site_col2", I32P),
        ("pent_row", I32P), ("pent_row2", I32P), ("eprog_ptr", I32P), ("eent_w", F64P), ("efac_ptr", I32P),
        ("efac_row", I32P), ("term_coef", F64P), ("term_body", I32P), ("term_ls", I32P), ("color_ptr", I32P),
        ("color_sites", I32P), ("site_has_l1", U8P), ("site_active", U8P),
    ]


class RunParams(C.Structure):
    _fields_ = [
        ("nsweeps", C.c_int64), ("or_per_metropolis", C.c_int32), ("exchange", C.c_int32),
        ("exchange_interval", C.c_int64), ("adapt_interval", C.c_int64), ("adapt_target", C.c_double),
        ("renorm_interval", C.c_int64), ("measure_interval", C.c_int64), ("lanes_per_site", C.c_int32),
        ("mode", C.c_int32), ("phase_done", C.c_int64), ("phase_total", C.c_int64), ("kernel", C.c_int32),
        ("proposals", C.c_int32), ("rep_replicas", C.c_int32), ("rep_threads_per_item", C.c_int32),
        ("rep_prefetch", C.c_int32),
    ]


class ScemcError(RuntimeError):
    """A non-zero status from libscemc_cuda.so."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[scemc status {code}] {msg}")
        self.code = code


class ScemcArgumentError(ScemcError, ValueError):
    """ArgumentError / DimensionMismatch equivalents (status SCEMC_ERR_ARG)."""


_lib = None

# (name, restype, argtypes) for every entry point of include/scemc.h
SIGNATURES = [
    ("scemc_last_error", C.c_int32, [C.c_char_p, C.c_size_t]),
    ("scemc_version", C.c_int32, []),
    ("scemc_tables_create", C.c_int32, [C.POINTER(TablesDesc), C.POINTER(C.c_void_p)]),
    ("scemc_tables_destroy", C.c_int32, [C.c_void_p]),
    ("scemc_tables_stats", C.c_int32, [C.c_void_p, F64P, F64P, I64P]),
    ("scemc_tables_records", C.c_int32, [C.c_void_p, F64P]),
    ("scemc_chain_create", C.c_int32, [C.c_void_p, F64P, C.c_double, C.c_uint64, C.c_double, C.POINTER(C.c_void_p)]),
    ("scemc_chain_destroy", C.c_int32, [C.c_void_p]),
    ("scemc_metropolis_sweep", C.c_int32, [C.c_void_p, C.c_void_p, C.c_double, C.c_int32, I64P]),
    ("scemc_overrelaxation_sweep", C.c_int32, [C.c_void_p, C.c_void_p, C.c_double, C.c_int32, I64P, I64P]),
    ("scemc_run_sweeps", C.c_int32, [C.c_void_p, C.c_void_p, C.c_double, C.c_int64, C.c_int64, C.c_int32]),
    ("scemc_download", C.c_int32, [C.c_void_p, F64P, F64P, I64P, I64P]),
    ("scemc_upload", C.c_int32, [C.c_void_p, F64P, C.c_double]),
    ("scemc_set_step", C.c_int32, [C.c_void_p, C.c_double]),
    ("scemc_swap_payload", C.c_int32, [C.c_void_p, C.c_void_p]),
    ("scemc_total_energy", C.c_int32, [C.c_void_p, C.c_int32, F64P]),
    ("scemc_renormalize", C.c_int32, [C.c_void_p, F64P]),
    ("scemc_batch_create", C.c_int32, [C.c_int32, C.POINTER(C.c_void_p), I32P, F64P, F64P, U64P, F64P,
                                       C.POINTER(C.c_void_p)]),
    ("scemc_batch_destroy", C.c_int32, [C.c_void_p]),
    ("scemc_batch_size", C.c_int32, [C.c_void_p, I32P, I64P]),
    ("scemc_batch_set_betas", C.c_int32, [C.c_void_p, F64P]),
    ("scemc_batch_set_steps", C.c_int32, [C.c_void_p, F64P]),
    ("scemc_batch_run", C.c_int32, [C.c_void_p, C.POINTER(RunParams)]),
    ("scemc_batch_run_async", C.c_int32, [C.c_void_p, C.POINTER(RunParams)]),
    ("scemc_batch_sync", C.c_int32, [C.c_void_p]),
    ("scemc_batch_stream", C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("scemc_batch_upload", C.c_int32, [C.c_void_p, F64P, F64P]),
    ("scemc_host_register", C.c_int32, [C.c_void_p, C.c_int64]),
    ("scemc_batch_state_bytes", C.c_int32, [C.c_void_p, I64P]),
    ("scemc_batch_save_state", C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64]),
    ("scemc_batch_load_state", C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64]),
    ("scemc_host_unregister", C.c_int32, [C.c_void_p]),
    ("scemc_batch_profile", C.c_int32, [C.c_void_p, C.c_int32]),
    ("scemc_batch_kernel_time", C.c_int32, [C.c_void_p, F64P, I64P]),
    ("scemc_batch_launches", C.c_int32, [C.c_void_p, I64P]),
    ("scemc_energy_gradient", C.c_int32, [C.c_void_p, F64P, C.c_int32, F64P]),
    ("scemc_batch_set_learned", C.c_int32, [C.c_void_p, C.c_void_p, I32P, C.c_int32]),
    ("scemc_batch_fetch_record_ratio", C.c_int32, [C.c_void_p, F64P]),
    ("scemc_batch_site_coeffs", C.c_int32, [C.c_void_p, C.c_int32, F32P]),
    ("scemc_mlp_create", C.c_int32, [C.c_uint64, C.c_int32, C.POINTER(C.c_void_p)]),
    ("scemc_mlp_destroy", C.c_int32, [C.c_void_p]),
    ("scemc_mlp_get_params", C.c_int32, [C.c_void_p, F32P]),
    ("scemc_mlp_set_params", C.c_int32, [C.c_void_p, F32P]),
    ("scemc_mlp_forward", C.c_int32, [C.c_void_p, F32P, C.c_int64, F32P]),
    ("scemc_mlp_loss_grad", C.c_int32, [C.c_void_p, F32P, F32P, C.c_int64, F64P, F32P]),
    ("scemc_mlp_train", C.c_int32, [C.c_void_p, F32P, F32P, C.c_int64, C.c_int32, C.c_int32, C.c_double, C.c_uint64,
                                    F64P]),
    ("scemc_batch_autotune", C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, I32P, I32P, I32P, I32P, F64P]),
    ("scemc_batch_download", C.c_int32, [C.c_void_p, F64P, F64P, I32P, I64P, I64P, F64P, F64P]),
    ("scemc_batch_reset_counters", C.c_int32, [C.c_void_p]),
    ("scemc_batch_fetch_measurements", C.c_int32, [C.c_void_p, F64P, C.c_int64, I64P, I32P]),
    ("scemc_batch_record", C.c_int32, [C.c_void_p, C.c_int32]),
    ("scemc_batch_record_slot", C.c_int32, [C.c_void_p, C.c_int32, C.c_int32]),
    ("scemc_batch_fetch_record", C.c_int32, [C.c_void_p, C.c_int32, F32P, F64P, F32P, U8P]),
    ("scemc_color_sites", C.c_int32, [C.c_int32, I32P, I32P, I32P, I32P, U8P, I32P, I32P]),
    ("scemc_selftest_barrier_timeout", C.c_int32, [C.c_int64]),
    ("scemc_l2_probe", C.c_int32, [C.c_int64, C.c_int32, F64P]),
    ("scemc_total_energy_static", C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
]


def lib() -> C.CDLL:
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python scemontecarlo.jl_b200/build.py` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib().scemc_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code: int) -> None:
    if code != OK:
        msg = last_error()
        if code == ERR_ARG:
            raise ScemcArgumentError(code, msg)
        raise ScemcError(code, msg)


def ptr(a: np.ndarray, ctype):
    """Pointer to the data of a C-contiguous numpy array (kept alive by the caller)."""
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))
