"""Shared test setup: markers, import paths, and the two builds (the FP64 oracle
and libscemc_cuda.so) the tests need."""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _builds():
    import oracle  # noqa: F401  (oracle/oracle.py)
    oracle.build()
    sys.path.insert(0, str(ROOT / "scemontecarlo.jl_b200"))
    import build as scemc_build  # scemontecarlo.jl_b200/build.py
    sys.path.pop(0)
    scemc_build.build()
    yield


@pytest.fixture(scope="session")
def gpu():
    if not _gpu_available():
        pytest.skip("no CUDA device")
    return True
