"""Shared test set-up.

Tests marked ``gpu`` need a CUDA device and call the product through its C
ABI (``swfwi_b200/libswfwi_b200.so``); the rest run on CPU and check the
oracle against the golden fixtures, the host logic, and the library's
exported symbols.
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
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="session")
def ref():
    """The compiled reference (oracle/_ref); built here when the reference
    tree is present, skipped where it is neither built nor buildable."""
    import oracle
    if not oracle.available() and oracle.reference_tree():
        oracle.build()
    if not oracle.available():
        pytest.skip("oracle/_ref not built")
    return oracle.RefLib()


@pytest.fixture(scope="session")
def fdo():
    import oracle
    if not os.path.exists(os.path.join(oracle.REF_DIR, "libfd_oracle.so")):
        if oracle.reference_tree():
            oracle.build()
        else:
            pytest.skip("oracle/_ref not built")
    return oracle.FdOracle()


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import swfwi_b200
    swfwi_b200.lib()   # fails loudly when the library is missing
    return torch
