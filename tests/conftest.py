"""Shared test setup: the `gpu` marker, import paths, and fixtures."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

PKG_NAME = "webgpu-mpm-based-snow-simulation_b200"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def import_pkg():
    return importlib.import_module(PKG_NAME)


@pytest.fixture(scope="session")
def pkg():
    return import_pkg()


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle  # noqa: E402  (oracle/oracle.py, test infrastructure)
    oracle.build()
    return oracle


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu(pkg):
    """Skips unless a GPU is present; builds libmpm.so if needed."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    from importlib import import_module
    import_module(PKG_NAME + ".build").build()
    return pkg
