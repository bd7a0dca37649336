"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and call the
product through its C ABI; everything else runs on the CPU."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a library)")


@pytest.fixture(scope="session")
def ctx():
    import horkxg_b200 as hb
    c = hb.Context(0)
    yield c
    c.close()
