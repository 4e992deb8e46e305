"""Shared test set-up: the `gpu` marker, the package loader and helpers.

The package directory is ``wrt-project_b200`` (not an importable name), so it
is loaded here under the module name ``wrt_b200``.  ``oracle`` (the CPU
checker) is imported from the repository root.
"""
import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "wrt-project_b200"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    if "wrt_b200" in sys.modules:
        return sys.modules["wrt_b200"]
    spec = importlib.util.spec_from_file_location(
        "wrt_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrt_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


wrt = load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100)")


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def rel_max(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def ctx():
    c = wrt.Context(0)
    yield c
    c.close()
