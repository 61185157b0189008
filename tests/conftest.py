import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle's C restatement and libjci if they are absent (the
    build entry point compiles them; a fresh checkout gets them here)."""
    from oracle import oracle as orc
    if not os.path.exists(orc.ORACLE_SO):
        orc.build(ref=False)
    from jayci_b200 import LIBPATH, build
    if not os.path.exists(LIBPATH):
        build.build()
    yield
