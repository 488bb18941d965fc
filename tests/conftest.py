"""Shared test set-up.

Markers:
  gpu -- needs a CUDA device (B200); deselect with -m "not gpu".

The CPU oracle (oracle/) is test infrastructure: tests build and load it here
as the checker.  The CUDA library is built by __graft_entry__.build() or on
first use by bajo_b200.build.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA device")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="session")
def lib():
    from bajo_b200 import build as B
    B.build()
    from bajo_b200 import _lib
    return _lib.load()
