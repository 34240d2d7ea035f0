"""Shared pytest configuration.

Markers
  gpu  -- needs a CUDA device; these are the parity tests proper and go
          through libfamrdp_cuda.so's C ABI.  Run with ``-m gpu`` on a B200;
          ``-m "not gpu"`` runs the oracle, host-logic and ABI-surface tests.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference's tolerance fixtures (tests/conftest.py:7-13 of famrdp_jax).
RTOL = 1e-12
ATOL_STRICT = 1e-13


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def rtol():
    return RTOL


@pytest.fixture(scope="session")
def atol_strict():
    return ATOL_STRICT


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from famrdp_jax_b200 import _capi
    _capi.lib()  # fail loudly if the library is missing
    return torch.device("cuda", 0)
