"""Shared test setup: the gpu marker, the package (its directory name is not a
Python identifier, so it is loaded by path as ``pfs_b200``) and the oracle."""
from __future__ import annotations

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "particle-fluid-simulation_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def load_package():
    if "pfs_b200" in sys.modules:
        return sys.modules["pfs_b200"]
    spec = importlib.util.spec_from_file_location(
        "pfs_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pfs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle  # noqa: WPS433
    return oracle


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def pfs():
    return load_package()


@pytest.fixture(scope="session")
def ora():
    return load_oracle()


@pytest.fixture(scope="session")
def cuda_device():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return 0
