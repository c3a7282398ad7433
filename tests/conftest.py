import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def astra():
    """The product package (directory name is not an identifier)."""
    return importlib.import_module("astra-toolbox_b200")


@pytest.fixture(scope="session")
def geo():
    return importlib.import_module("astra-toolbox_b200.geometry")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    return oracle


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
