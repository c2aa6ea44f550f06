import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line(
        "markers", "slow: minutes of GPU time each (full solves at the "
                   "precision-table sizes); run only with LIBPT_SLOW_TESTS=1")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if not os.environ.get("LIBPT_SLOW_TESTS"):
        slow = pytest.mark.skip(reason="slow: set LIBPT_SLOW_TESTS=1")
        for it in items:
            if "slow" in it.keywords:
                it.add_marker(slow)
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
