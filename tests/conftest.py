"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built extension")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ff_lib():
    from firefly_b200 import build as B
    B.build()
    import firefly_b200 as ff
    return ff.lib()


@pytest.fixture(scope="session")
def oracle():
    from oracle import ffo
    ffo.build()
    ffo.load()
    return ffo


@pytest.fixture(scope="session")
def ctx(ff_lib):
    import firefly_b200 as ff
    c = ff.Context(0)
    yield c
    c.close()


def cpu_threads() -> int:
    return max(1, min(64, os.cpu_count() or 1))
