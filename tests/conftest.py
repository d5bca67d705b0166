"""pytest configuration: the `gpu` marker, import paths and shared fixtures."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle and, when nvcc is present and the sources are newer, the
    CUDA library (on a GPU host the prebuilt .so files are used as shipped)."""
    from oracle import oracle
    from aperi_mech_b200 import build

    oracle.build()
    if build.stale():
        build.build()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def capi_lib():
    from aperi_mech_b200 import build, capi

    build.build()
    return capi.load()


@pytest.fixture(scope="session")
def gpu(capi_lib):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    torch.cuda.init()
    return torch.device("cuda:0")
