"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def engine():
    import ymc3d_b200
    from ymc3d_b200 import build
    build.build()
    ymc3d_b200.lib()
    return ymc3d_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    from oracle import build
    build.build()
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def table(engine):
    return engine.default_table()


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
