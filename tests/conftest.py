import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Make sure the oracle and the CUDA library exist (built in-tree)."""
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build(with_ref=False)
    lib = os.path.join(ROOT, "hptt_b200", "libhptt_cuda.so")
    if not os.path.exists(lib):
        from hptt_b200 import build as b
        b.build()
    yield
