"""Shared test setup: the `gpu` marker, and loaders for the product package
(a folder whose name is not a Python identifier) and for the oracle."""
from __future__ import annotations

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "xray-directional-reconstruction_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_xr():
    """Import the product package xray-directional-reconstruction_b200 as `xrd`."""
    if "xrd" in sys.modules:
        return sys.modules["xrd"]
    spec = importlib.util.spec_from_file_location("xrd", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["xrd"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def xr():
    return load_xr()


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_ir_small.npz"))


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
