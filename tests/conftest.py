"""Test configuration: the `gpu` marker, import paths and shared helpers.

CPU tests (`-m "not gpu"`) check the oracle against the reference's known
answers and the golden fixtures produced by the compiled reference operator
code, and that the CUDA library loads with every C-ABI symbol.  GPU tests
(`-m gpu`) are the parity tests proper: they call the B200 backend through its
C ABI and compare with the oracle on the same seeded inputs.
"""
import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
PKG_DIR = REPO / "carousel-phase-retrieval-algorithm_b200"
for p in (str(PKG_DIR), str(REPO / "oracle"), str(REPO)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the backend through its C ABI")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda:0")
