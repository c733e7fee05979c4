"""Shared test setup: the `gpu` marker, import paths for the CUDA binding and the oracle.

Tests marked `gpu` need a CUDA device and the built `libks_b200.so`; everything else runs on the
CPU (the oracle, the host logic and the C-ABI surface)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "atomic-sandbox_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and the built CUDA library")


@pytest.fixture(scope="session")
def oracle():
    import ks_oracle
    ks_oracle.set_threads(min(8, os.cpu_count() or 1))
    return ks_oracle


@pytest.fixture(scope="session")
def ks():
    import ks_b200
    return ks_b200
