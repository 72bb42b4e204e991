"""Shared test set-up: markers, import paths, and the CPU checkers (oracle/)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def bits(a):
    """Bit pattern view for exact comparisons (distinguishes -0.0 and NaN payloads)."""
    a = np.ascontiguousarray(a)
    return a.view(np.int64) if a.dtype == np.float64 else a


def assert_bits_equal(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if not np.array_equal(bits(a), bits(b)):
        d = np.abs(a - b)
        i = np.unravel_index(np.nanargmax(d), d.shape) if np.isfinite(d).any() else None
        raise AssertionError("%s differs in %d entries; max |diff| %g at %s (%r vs %r)" % (
            what, int((bits(a) != bits(b)).sum()), np.nanmax(d), i, a[i] if i else None, b[i] if i else None))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import refpy
    refpy.build_oracle()
    return refpy
