import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle libraries (and libsphgpu.so when sources changed)."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    from graphics_b200.csrc import build as b  # noqa
    b.build()
    yield
