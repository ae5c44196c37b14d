"""Shared fixtures: the package (loaded from its directory), the oracle and
the `gpu` marker.  Tests marked gpu need an sm_100 device; the rest run on
any machine."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "4hetddft-isotropic-bohmian_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")


def load_pkg():
    name = "he4b200"
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
    import oracle  # noqa: E402
    oracle.build()
    return oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def ora():
    load_pkg()
    return load_oracle()
