import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs through the C ABI of libtomo_b200.so)")
    config.addinivalue_line("markers", "slow: larger parity cases")


@pytest.fixture(scope="session")
def tomo():
    """The product library, built in-tree if needed.  No fallback: a GPU test fails if it
    cannot be built or loaded."""
    import seismic_tomography_3d_b200 as tomo_pkg
    from seismic_tomography_3d_b200 import build

    build.build()
    tomo_pkg.load_library()
    return tomo_pkg


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle
