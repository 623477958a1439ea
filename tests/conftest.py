"""Shared pytest setup: import paths, the ``gpu`` marker and small seeded inputs.

Lanes (mirroring the reference's CPU / GPU split, tests/conftest.py:19-43 there):
* ``-m "not gpu"`` — oracle against the reference's known answers and golden fixtures, host
  logic, and that the C-ABI library loads and exports every declared symbol;
* ``-m gpu`` — parity of the CUDA path against the oracle, called through the C ABI.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "metal-singlecell_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def mixture_10k():
    from msc_b200 import synth
    X, params = synth.plain_10k()
    return X, params
