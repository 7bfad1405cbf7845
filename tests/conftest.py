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
