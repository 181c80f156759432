import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs the CUDA path)")


@pytest.fixture(scope="session")
def built():
    """Builds the product libraries and the oracle once per session."""
    from nicp_b200 import build
    from oracle import oracle
    build.build_all()
    oracle.build()
    return True


@pytest.fixture(scope="session")
def ctx(built):
    from nicp_b200 import Context
    c = Context.default()
    yield c
