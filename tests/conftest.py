"""Shared test set-up: import paths and the `gpu` marker.

`-m "not gpu"` runs the oracle pinning, host logic and C-ABI load/export tests on CPU;
`-m gpu` runs the parity tests through the C ABI on a CUDA device.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "vajra-opt_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through libvajra_pdhg.so")


def cuda_device_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not cuda_device_present():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    import torch
    return torch.device("cuda:0")
