"""Test configuration: the `gpu` marker, shared helpers and fixtures.

`-m "not gpu"` runs the oracle / host-logic / ABI tests on the CPU;
`-m gpu` runs the parity tests of the CUDA path against the oracle.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def rel_l2(a, b, floor=0.0):
    """||a - b||_2 / max(||b||_2, floor)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / max(nb, floor, 1e-300)


def max_var_rel_l2(a, b, rel_floor=1e-12):
    """max over variables (axis 0) of the relative L2 difference; a variable
    whose reference norm is tiny is measured against rel_floor x the largest
    variable norm."""
    top = max(np.linalg.norm(b[n].ravel()) for n in range(b.shape[0]))
    return max(rel_l2(a[n], b[n], floor=rel_floor * top) for n in range(b.shape[0]))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.load()
    return oracle
