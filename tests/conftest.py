"""Test configuration: the ``gpu`` marker, and the repository root on sys.path."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        have_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def no_device_errors(request):
    """GPU tests leave no bounded-wait error bits behind in the backend."""
    yield
    if "gpu" in request.keywords:
        import torch

        if torch.cuda.is_available():
            from mpifield_b200 import _lib

            assert _lib.device_errors(clear=True) == 0
