"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on any machine: the oracle against the golden fixtures (and against
the reference build when it is present), host-side logic, and the C-ABI library's
exports.  `-m gpu` needs a B200 and the built library; those tests are the parity tests
proper and call the CUDA path through the C ABI.
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
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built CUDA library")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.fixture(scope="session")
def gpu():
    """The CUDA library, loaded; fails (does not skip) when the GPU path is unusable, so a
    GPU run can never pass on a fallback."""
    import imagestack_b200 as ib
    assert ib.device_count() >= 1, "no sm_100 device visible to libpermgpu"
    return ib
