"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on any host (oracle vs golden vectors, host logic, the
C-ABI library's exports); `-m gpu` needs a CUDA device and calls the CUDA
path through the C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "apss-cuda_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def gpu_ctx():
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    import cuapss
    with cuapss.Context() as c:
        yield c
