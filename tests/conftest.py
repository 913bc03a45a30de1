import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    """Builds the CPU oracle (and, where the reference tree is mounted, the
    reference library) once per session."""
    import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def gpu_lib():
    """Builds libpu_dycore.so if it is older than its sources and loads it."""
    from porturb_b200 import build, capi
    build.build()
    return capi.load()
