import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: full-size configuration")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (and the product library when missing) once per session."""
    import oracle
    oracle.lib()
    from coolfluid3_b200 import build
    if not os.path.exists(build.LIB):
        build.build(quiet=True)
