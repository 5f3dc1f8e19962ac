"""Shared test setup: the ``gpu`` marker, oracle build and GPU helpers."""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libeman2_b200.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    from oracle import oracle
    oracle.build(ref=True)
    yield


def has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Skips nothing: a GPU test on a box without a GPU fails loudly."""
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    from eman2_b200 import _lib
    _lib.load()
    return torch.device("cuda:0")
