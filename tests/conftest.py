"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu() -> bool:
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
def oracle():
    from oracle.oracle import Restated, build

    build()
    return Restated()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, reference_available

    if not reference_available():
        pytest.skip("reference oracle library not built")
    return Reference()


@pytest.fixture(scope="session")
def capi():
    from vbcsr_b200 import _capi

    return _capi.load()


@pytest.fixture(scope="session")
def dev():
    import torch

    torch.cuda.init()
    return torch.device("cuda:0")


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)
