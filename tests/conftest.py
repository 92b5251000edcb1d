import os
import sys

import pytest

# the oracle's OpenMP threads sleep between parallel regions instead of
# spinning, leaving the cores to OpenBLAS where a check uses it (set before
# any OpenMP runtime is loaded)
os.environ.setdefault("OMP_WAIT_POLICY", "passive")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    """One lapw1gpu context on cuda:0 for the GPU tests."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    from hack_wein2k_b200 import lapw1gpu
    c = lapw1gpu.Context(0)
    yield c
    c.close()
