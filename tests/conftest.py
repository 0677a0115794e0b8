"""Test configuration: the `gpu` marker and session-wide builds of the native libraries."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def native_libs():
    """Builds libwgpt.so and the oracle when their sources changed (no-op otherwise)."""
    from webgpuraytracer_b200 import build
    import oracle

    build.build()
    oracle.build()
    yield
