import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "reference: needs the compiled reference (oracle/_ref)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """The CPU checkers and the CUDA library must exist; build them if not."""
    from xdem_b200 import build as b
    import oracle
    if not os.path.exists(oracle.PORT_LIB):
        oracle.build()
    if not os.path.exists(b.LIB):
        b.build()
    yield
