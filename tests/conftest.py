import os
import sys

import pytest

TESTS = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(TESTS)
for p in (ROOT, TESTS):      # the package and oracle; test modules that share helpers
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the kernels through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Compile libpsb.so and the oracle if they are missing or stale (nvcc
    cross-compiles without a GPU)."""
    from psb_project_b200 import build as B
    B.build()
    import oracle
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build(with_reference=False)
    yield
