"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built
libtomo_b200.so; everything else runs on the CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and libtomo_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref_engine():
    """The reference INT3 engine built from the reference sources, when present."""
    from oracle import build
    from oracle.oracle import RefEngine
    path = build.build_ref()
    if path is None or not Path(path).exists():
        pytest.skip("reference engine library not available")
    return RefEngine(path)
