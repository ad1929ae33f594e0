"""Shared fixtures.  The engine package lives in the hyphenated directory
total-viewsheds_b200/ and is loaded here under the module name
total_viewsheds_b200; the CPU oracle (test infrastructure) is oracle/oracle.py."""

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "total-viewsheds_b200"
GOLDEN = ROOT / "tests" / "golden" / "reference_vectors.json"


def load_package():
    if "total_viewsheds_b200" in sys.modules:
        return sys.modules["total_viewsheds_b200"]
    spec = importlib.util.spec_from_file_location(
        "total_viewsheds_b200", PKG_DIR / "__init__.py",
        submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["total_viewsheds_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # noqa: E402
    return oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libtvs_cuda.so")


@pytest.fixture(scope="session")
def tvs():
    from_pkg = load_package()
    return from_pkg


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()


@pytest.fixture(scope="session")
def golden():
    return json.loads(GOLDEN.read_text())


@pytest.fixture(scope="session")
def synth():
    load_package()
    import total_viewsheds_b200.dem_synth as ds
    return ds


@pytest.fixture(scope="session")
def bt():
    load_package()
    import total_viewsheds_b200.bt_io as b
    return b


def f32(values):
    return np.array(values, dtype=np.float32)
