"""Test configuration: the `gpu` marker and one-time builds of the oracle and
the CUDA library (both no-ops when up to date)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from oracle import build_oracle
    build_oracle.build_oracle()
    build_oracle.build_ref()
    build_oracle.build_ref_init()
    from emu_b200 import build
    if os.path.exists("/usr/local/cuda/bin/nvcc") or not os.path.exists(build.LIB):
        build.build()
    yield
