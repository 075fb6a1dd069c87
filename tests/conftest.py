import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests against the oracle")
    config.addinivalue_line("markers", "slow: longer CPU runs")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle (test infrastructure) once per session."""
    from oracle import build as ob
    ob.build()
    yield
