import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def gpu_lib():
    """Build (if stale) and load libcismgpu.so; the GPU tests fail loudly without it."""
    from cism_b200 import build, load_library
    build.build()
    return load_library()
