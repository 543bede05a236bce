import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through the C ABI")


@pytest.fixture(scope="session")
def golden():
    """Reference-generated fixtures: {B: npz} (tests/golden/make_golden.py)."""
    out = {}
    for B in (2, 4, 8, 16):
        out[B] = dict(np.load(os.path.join(GOLDEN, f"ref_B{B}.npz")))
    return out


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def lib():
    import pfsoftlib_b200

    return pfsoftlib_b200.load()
