"""Build recipe of libscemc_cuda.so (sm_100a only).

The library is compiled in-tree next to this file so that it travels with the
repository; it links the CUDA runtime statically, so loading it needs only the
driver (and no driver at all for the host-only entry points).
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc" / "scemc.cu"
HDRS = [PKG / "csrc" / "scemc_device.cuh", ROOT / "include" / "scemc.h"]
LIB = PKG / "libscemc_cuda.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
    "-diag-suppress", "177",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libscemc_cuda.so")


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [SRC, *HDRS])


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile libscemc_cuda.so if it is missing or older than its sources."""
    if not force and not stale():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, f"-I{ROOT / 'include'}", "-o", str(tmp), str(SRC)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
