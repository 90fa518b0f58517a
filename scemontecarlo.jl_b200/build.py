"""Build recipe of libscemc_cuda.so (sm_100a only).

The library is compiled in-tree next to this file so that it travels with the
repository; it links the CUDA runtime statically, so loading it needs only the
driver (and no driver at all for the host-only entry points). The two
translation units (the sweep library and the learned-proposal network) compile in
parallel and link into one shared object.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import pathlib
import shutil
import subprocess

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
SRCS = [PKG / "csrc" / "scemc.cu", PKG / "csrc" / "learned.cu"]
HDRS = [PKG / "csrc" / "scemc_device.cuh", PKG / "csrc" / "umma.cuh", PKG / "csrc" / "vmf.cuh",
        PKG / "csrc" / "mlp.h", ROOT / "include" / "scemc.h"]
LIB = PKG / "libscemc_cuda.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "177"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libscemc_cuda.so")


STAMP = LIB.with_name(LIB.name + ".srchash")


def source_hash(extra=()) -> str:
    """SHA-256 over the sources, headers and compiler flags the library is built from."""
    h = hashlib.sha256()
    for p in [*SRCS, *HDRS]:
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(" ".join([*NVCC_FLAGS, *extra]).encode())
    return h.hexdigest()


def stale() -> bool:
    """True unless the library exists and its stamp holds the current source hash
    (a prebuilt library from other sources is rebuilt, whatever its mtime)."""
    if not LIB.exists() or not STAMP.exists():
        return True
    return STAMP.read_text().strip() != source_hash()


def _compile(src: pathlib.Path, obj: pathlib.Path, extra) -> subprocess.CompletedProcess:
    cmd = [nvcc(), *NVCC_FLAGS, *extra, f"-I{ROOT / 'include'}", "-c", "-o", str(obj), str(src)]
    return subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False, extra=(), out: pathlib.Path | None = None) -> pathlib.Path:
    """Compile libscemc_cuda.so if it is missing or was built from other sources."""
    out = out or LIB
    if out == LIB and not force and not stale():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = [objdir / (s.stem + ".o") for s in SRCS]
    with cf.ThreadPoolExecutor(len(SRCS)) as ex:
        res = list(ex.map(lambda so: _compile(so[0], so[1], list(extra)), zip(SRCS, objs)))
    for r in res:
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        if verbose:
            print(r.stdout + r.stderr)
    tmp = out.with_suffix(".so.tmp")
    link = subprocess.run([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)],
                          capture_output=True, text=True)
    if link.returncode != 0:
        raise RuntimeError("link failed:\n" + link.stdout + link.stderr)
    os.replace(tmp, out)
    if out == LIB:
        STAMP.write_text(source_hash(extra) + "\n")
    return out


if __name__ == "__main__":
    print(build(force=True, verbose=True))
