"""Test configuration: registers the ``gpu`` marker and import paths.

``-m "not gpu"`` runs everything that needs no GPU (oracle known-answer
checks, host logic, C-ABI symbol checks); ``-m gpu`` runs the parity tests
of the CUDA engine against the oracle on a B200.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
