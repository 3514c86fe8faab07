"""Shared fixtures.  The package directory is named inspire-rs_b200 (not a
Python identifier), so it is imported by path as `inspire_rs_b200`."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_package():
    if "inspire_rs_b200" in sys.modules:
        return sys.modules["inspire_rs_b200"]
    pkg_dir = os.path.join(ROOT, "inspire-rs_b200")
    spec = importlib.util.spec_from_file_location(
        "inspire_rs_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["inspire_rs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    import oracle
    return oracle


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle
