import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU; run with -m gpu")


@pytest.fixture(scope="session")
def backend():
    from cumulus3d_b200.patchstereo import PatchMatchBackend
    return PatchMatchBackend(0, math="parity")


@pytest.fixture(scope="session")
def backend_fast():
    from cumulus3d_b200.patchstereo import PatchMatchBackend
    return PatchMatchBackend(0, math="fast")
