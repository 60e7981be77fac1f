"""Shared pytest setup: the ``gpu`` marker and import paths.

Tests marked ``gpu`` need a CUDA device and the built ``librakali.so``; the
rest run on CPU (oracle known-answer tests, config/host logic, C-ABI symbol
checks, gloo multi-process tests).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")
    config.addinivalue_line("markers", "slow: long CPU oracle run (seconds)")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover - torch missing
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc
    orc.lib()
    return orc
