"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "multi-gpu-sorting_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_mgs():
    """Imports the engine's Python binding (multi-gpu-sorting_b200/mgs.py)."""
    if "mgs" in sys.modules:
        return sys.modules["mgs"]
    spec = importlib.util.spec_from_file_location("mgs", os.path.join(PKG, "mgs.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["mgs"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def mgs():
    return load_mgs()


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def ctx(mgs):
    c = mgs.Context(0)
    yield c
    c.close()
