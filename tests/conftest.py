"""Shared pytest configuration.

* registers the `gpu` marker (tests that need a CUDA device);
* makes the oracle (`oracle/ffcm_oracle.py`) and the product package
  (`ffcm.jl_b200/`, imported under the name `ffcm_b200`) importable;
* restates the reference's shared fixtures (test/test_utilities.jl).
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))


def load_product():
    """Import `ffcm.jl_b200/` as the package `ffcm_b200`."""
    if "ffcm_b200" in sys.modules:
        return sys.modules["ffcm_b200"]
    pkg = ROOT / "ffcm.jl_b200"
    spec = importlib.util.spec_from_file_location(
        "ffcm_b200", pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ffcm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def ffcm():
    return load_product()


@pytest.fixture(scope="session")
def oracle():
    import ffcm_oracle
    return ffcm_oracle
