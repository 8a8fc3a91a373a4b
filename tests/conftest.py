import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("ray-tracer_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels through the C ABI")
    # An assertion inside a ctypes callback is otherwise swallowed; make it fail the test.
    config.addinivalue_line("filterwarnings", "error::pytest.PytestUnraisableExceptionWarning")


@pytest.fixture(scope="session")
def ctx():
    import rtg

    c = rtg.Context(0)  # fails loudly without a GPU or without librtg.so
    yield c
    c.close()
