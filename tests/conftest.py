import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU; parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle.get()


@pytest.fixture(scope="session")
def golden_chem():
    return dict(np.load(os.path.join(GOLDEN, "gri30_chem_golden.npz")))


@pytest.fixture(scope="session")
def golden_e2e():
    return dict(np.load(os.path.join(GOLDEN, "e2e_gri100.npz")))


def y_ok(Y_test, Y_ref, rel=1e-4, abs_=1e-10):
    """Per-entry mass-fraction gate: |dY| <= max(rel*|Y_ref|, abs_)."""
    return np.abs(Y_test - Y_ref) <= np.maximum(rel * np.abs(Y_ref), abs_)


@pytest.fixture(scope="session")
def golden_enthalpy():
    return dict(np.load(os.path.join(GOLDEN, "enthalpy_ref.npz")))

