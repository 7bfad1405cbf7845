import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA device (B200)")


PKG_DIR = os.path.join(ROOT, "shallow-water_b200")


def load_package():
    """Import the shallow-water_b200 directory as the package ``shallow_water_b200``."""
    import importlib.util
    if "shallow_water_b200" in sys.modules:
        return sys.modules["shallow_water_b200"]
    spec = importlib.util.spec_from_file_location(
        "shallow_water_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["shallow_water_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_cache = {}


def golden(group):
    """Golden vectors of one reference module (see tests/golden/make_golden.py)."""
    if group not in _cache:
        _cache[group] = dict(np.load(os.path.join(GOLDEN, group + ".npz")))
    return _cache[group]


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc
    orc.lib()
    return orc


@pytest.fixture(scope="session")
def sw():
    return load_package()
