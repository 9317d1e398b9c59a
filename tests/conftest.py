"""pytest configuration: the `gpu` marker and one-time native builds."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def native_builds():
    """Builds the product library, the CPU oracle and the product-linked scene
    driver when missing or stale (rfsyn's own sources are built into
    oracle/_ref only where they exist)."""
    from rfsyn_b200 import build as b
    import oracle

    b.build()
    oracle.build(ref=True)
    oracle.build_driver()
    yield
