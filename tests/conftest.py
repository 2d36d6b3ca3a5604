"""Shared test set-up: import paths, the gpu marker, fixture locations.

GPU tests (``-m gpu``) call the product through the C ABI (libfemmgpu.so) and check
it against the CPU oracle (oracle/, test infrastructure only).  CPU tests check the
oracle against the reference's golden vectors, the host logic, and that the library
loads and exports every symbol of include/femm_gpu.h.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("femm-gpu_b200", "oracle"):
    path = os.path.join(ROOT, sub)
    if path not in sys.path:
        sys.path.insert(0, path)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return True
