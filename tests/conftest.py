import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "modlin-rs_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

M61 = 2305843009213693951


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def O():
    """The CPU oracle (test infrastructure)."""
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def built_lib():
    """Path of libmodlin_gpu.so, building it (nvcc cross-compile) if needed."""
    so = os.path.join(PKG, "libmodlin_gpu.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-j8", "-C", PKG], check=True)
    return so


@pytest.fixture(scope="session")
def M(built_lib):
    """The product binding (modlin package over the C ABI)."""
    import modlin
    return modlin
