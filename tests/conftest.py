import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libbfm.so")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds libbfm.so (nvcc cross-compiles without a GPU) and the oracle once per session."""
    from pscbfm_b200 import build as B
    B.build()
    from oracle import oracle as O
    if not os.path.exists(O.LIB):
        O.build()
