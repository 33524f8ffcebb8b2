"""Shared fixtures: the engine package (ctypes over libwfb200.so) and the oracle bindings."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "graphics-book-tutorials_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def load_engine():
    if "wfb200" in sys.modules:
        return sys.modules["wfb200"]
    spec = importlib.util.spec_from_file_location("wfb200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wfb200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import oracle  # noqa: E402
    return oracle


@pytest.fixture(scope="session")
def wfb():
    mod = load_engine()
    mod.load_library()
    return mod


@pytest.fixture(scope="session")
def orc():
    return load_oracle()


@pytest.fixture(scope="session")
def ref(orc):
    if not orc.reference_available():
        pytest.fail("oracle/_ref/libwfref.so is missing: build it with `make -C oracle` where the reference exists")
    return orc
