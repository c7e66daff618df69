"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU check")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def cep():
    """The product package; builds the CUDA library if it is missing."""
    mod = importlib.import_module("2ddrugsimulation_b200")
    if not mod.LIB_PATH.exists():
        from importlib import import_module
        import_module("2ddrugsimulation_b200.build").build()
    return mod


@pytest.fixture(scope="session")
def gpu(cep):
    """Fails loudly (no skip) when a GPU test runs without a device."""
    n = cep.device_count()
    assert n > 0, "GPU test collected but no CUDA device is visible"
    return n
