"""Test configuration: the `gpu` marker, import paths, and shared fixtures.

Tests marked `gpu` need a CUDA device and the built librivet_me.so; the
rest run on the CPU (the oracle, the host-side logic, the library's
exported symbols).
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def ms():
    """One MotionSearch context for the GPU tests of a session."""
    import rivet_h26x_codecs_b200 as rme
    ctx = rme.MotionSearch(0)
    yield ctx
    ctx.close()
