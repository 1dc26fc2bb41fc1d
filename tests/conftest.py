"""Shared test setup: the `gpu` marker, package / oracle loading, fixtures."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "rw-spgemm_b200"


def load_package():
    """Import the package that lives in the hyphenated directory rw-spgemm_b200/."""
    if "rw_spgemm_b200" in sys.modules:
        return sys.modules["rw_spgemm_b200"]
    spec = importlib.util.spec_from_file_location("rw_spgemm_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["rw_spgemm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if "tsg_oracle_py" in sys.modules:
        return sys.modules["tsg_oracle_py"]
    spec = importlib.util.spec_from_file_location("tsg_oracle_py", ROOT / "oracle" / "oracle.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tsg_oracle_py"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def tsg():
    return load_package()


@pytest.fixture(scope="session")
def gen():
    load_package()
    import rw_spgemm_b200.generators as g
    return g


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()


@pytest.fixture(scope="session")
def ctx(tsg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    c = tsg.Context(0)
    yield c
    c.close()
