"""Test configuration: the `gpu` marker, the package import (its directory name has a hyphen), and the
CPU oracle library (test infrastructure) built on demand."""
import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "riftphys-rust_b200")
ORACLE_LIB = os.path.join(ROOT, "oracle", "build", "liboracle_rphys.so")


def _import_pkg():
    if "riftphys_rust_b200" in sys.modules:
        return sys.modules["riftphys_rust_b200"]
    spec = importlib.util.spec_from_file_location("riftphys_rust_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["riftphys_rust_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


rp = _import_pkg()
import riftphys_rust_b200.scenes as scenes  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def oracle_lib():
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    return rp.Lib(ORACLE_LIB)


@pytest.fixture(scope="session")
def oracle():
    return oracle_lib()


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return rp.load_product()
