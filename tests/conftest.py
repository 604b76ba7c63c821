"""Test configuration: the ``gpu`` marker and shared fixtures.

``-m "not gpu"`` runs on any machine (oracle vs golden fixtures, host logic,
library symbols); ``-m gpu`` needs a CUDA device and the built library and
compares the library with the oracle and the golden fixtures.
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and libdfjk.so")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}_ref.npz")))


def golden_basis(g, prefix):
    from dftax_b200.basis import BasisData

    return BasisData(centers=g[f"{prefix}_centers"], exponents=g[f"{prefix}_exponents"],
                     coefficients=g[f"{prefix}_coefficients"], angular=g[f"{prefix}_angular"],
                     cart2sph=g[f"{prefix}_cart2sph"])


def unpack_tril(tril, n):
    out = np.zeros((n, n) + tril.shape[1:])
    a, b = np.tril_indices(n)
    out[a, b] = tril
    out[b, a] = tril
    return out


@pytest.fixture(scope="session")
def water_golden():
    return load_golden("water")


@pytest.fixture(scope="session")
def ch2_golden():
    return load_golden("ch2")
