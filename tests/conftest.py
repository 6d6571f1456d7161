"""Shared test set-up.

Markers: ``gpu`` -- needs a CUDA device (the parity tests proper, run on a
B200); everything else runs on the CPU.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def product_lib():
    """The in-tree libhydro_b200.so (built if missing; never a fallback)."""
    from hydro_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "hydro_b200", "csrc")], check=True)
    return _lib.load()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.oracle_lib()
    return O
