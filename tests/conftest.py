import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build libgpudb.so and the oracle once per session (no-op when up to date)."""
    from gpudbmetalcodegen_b200 import build_native
    from oracle import build_oracle
    build_native.build()
    build_oracle.build()


@pytest.fixture(scope="session")
def ctx():
    from gpudbmetalcodegen_b200.engine import Context
    c = Context(0)
    yield c
    c.close()
