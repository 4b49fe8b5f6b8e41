import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


def golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


@pytest.fixture(scope="session")
def gold():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = golden(name)
        return cache[name]
    return get


def fortran(a):
    """Golden matrices are stored column-major as (cols, rows): return the (rows, cols) view."""
    return np.asarray(a).T


def rel_entry_err(a, b):
    """max |a-b| / max(|b_ij|, max_row |b|): the entrywise rule used for nearfield parity."""
    a, b = np.asarray(a), np.asarray(b)
    rowmax = np.max(np.abs(b), axis=1, keepdims=True)
    denom = np.maximum(np.abs(b), rowmax)
    denom[denom == 0] = 1.0
    return float(np.max(np.abs(a - b) / denom))
