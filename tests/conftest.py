import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (run with -m gpu)")


@pytest.fixture(scope="session")
def oracle():
    """The CPU restatement (test infrastructure)."""
    from oracle import oracle as o

    o.build()
    return o


@pytest.fixture(scope="session")
def backend():
    """The CUDA backend on cuda:0; raises (fails the test) when the library or GPU is missing."""
    from continuum_liquid_b200 import build
    from continuum_liquid_b200.backend import Backend

    build.build_library()
    return Backend(0)
