import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs the CUDA library)")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the CUDA library in-tree once per session."""
    from oracle import oracle
    oracle.build()
    from mcv_sw_b200 import build
    build.build()
