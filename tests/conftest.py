import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "immsered-boundary_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def load_pkg():
    name = "immsered_boundary_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import pyoracle
    return pyoracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()


@pytest.fixture(scope="session")
def cuda_lib(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device")
    lib = pkg.ibgpu.lib()  # raises if the CUDA library is missing: no fallback
    torch.cuda.init()
    return lib
