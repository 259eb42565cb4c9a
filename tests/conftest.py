"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device (a B200); all
others run on the CPU against the oracle and the built libraries."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    build()
    return Oracle


def load_golden(dims):
    return np.load(os.path.join(GOLDEN, "ref_%dx%dx%d.npz" % tuple(dims)))


GOLDEN_GRIDS = [(16, 16, 16), (16, 24, 32)]
