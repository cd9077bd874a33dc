"""Shared test setup: the ``gpu`` marker and import paths.

Tests marked ``gpu`` need a CUDA device and the in-tree sm_100a library; the
rest run on the CPU (oracle against the golden fixtures, host-side logic, the
C-ABI library's exported symbols, multi-process ``gloo`` paths).
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a) and the built library")


@pytest.fixture(scope="session")
def golden():
    """Load a golden fixture by file name."""
    import numpy as np

    cache = {}

    def load(name):
        if name not in cache:
            cache[name] = dict(np.load(os.path.join(GOLDEN, name)))
        return cache[name]

    return load
