"""Test configuration: registers the ``gpu`` marker and puts the package and the
oracle on sys.path.

``-m "not gpu"`` runs on any machine (oracle vs golden vectors, host logic,
C-ABI exports); ``-m gpu`` tests need a CUDA device and call the CUDA library
through its C ABI, comparing against the CPU oracle.
"""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("boiling-sim_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libbsproj.so")


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    from boilingsim_b200 import _lib

    _lib.lib()  # raises if the library is missing: no fallback
    return torch.device("cuda:0")
