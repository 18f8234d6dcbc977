"""Test configuration: the `gpu` marker and shared fixtures.

CPU tests (``-m "not gpu"``) cover the oracle against the golden vectors
generated from the reference (``tests/golden/make_golden.py``), host logic,
and that libvoxfea loads and exports its C-ABI.  GPU tests call the CUDA path
through the C-ABI and compare it with the oracle / golden vectors.
"""

import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")


def golden(name):
    with np.load(os.path.join(GOLDEN, name), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def lib():
    from voxelsim_fea_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def gpu():
    """Skip-free guard: GPU tests require a working device and fail loudly otherwise."""
    from voxelsim_fea_b200 import backend
    assert backend.gpu_usable(), backend.gpu_status()
    return True
