"""Shared test set-up: import paths, the `gpu` marker, and on-demand builds of
the oracle (always) and of the product library (only when missing)."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import oracle.build as ob
    ob.build_oracle()
    if not (ROOT / "fvstuff_b200" / "libfvb.so").exists():
        from fvstuff_b200 import build as fb
        fb.build()
    yield


def have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
