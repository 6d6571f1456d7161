"""Shared test set-up.

Markers: ``gpu`` -- needs a CUDA device (the parity tests proper, run on a
B200); everything else runs on the CPU.
"""
import os
import subprocess
import sys

import numpy as np
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


@pytest.fixture(scope="session")
def reference_4096_200(oracle):
    """The 4096^2 centred blast's whole 200-step run by the reference's own
    C99/OpenMP code (oracle/_ref, compiled from the reference sources) on all
    host cores, computed once per session: (state, dt sequence, final t).
    Skips where the reference was not compiled."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the reference compiled from its sources) is not built: "
                    "the full-run tests need the reference itself")
    from hydro_b200 import make_params
    from _helpers import orc_from_H
    H = make_params(4096, 4096, testcase=0)
    ref = oracle.RefState(orc_from_H(oracle, H), 0)
    n, dts, t, _, _ = ref.run(200)
    u = ref.get()
    ref.close()
    assert n == 200
    return u, np.asarray(dts), t
