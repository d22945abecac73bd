"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built
native library; everything else runs on the CPU."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built native library")
    config.addinivalue_line("markers", "slow: takes more than ~10 s")


def _has_gpu():
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
def g118():
    from gpusim2grid_b200.synthetic import grid_by_name
    return grid_by_name("case118_synth", 0)


@pytest.fixture(scope="session")
def g2000():
    from gpusim2grid_b200.synthetic import grid_by_name
    return grid_by_name("case2000_synth", 0)


@pytest.fixture(scope="session")
def g6500():
    from gpusim2grid_b200.synthetic import grid_by_name
    return grid_by_name("case6500_synth", 0)


# tolerances: FP64 engine vs FP64 oracle (same algorithm, different sparse LU
# and summation order); mixed precision converges to the same 1e-8 mismatch,
# so its voltages differ from the FP64 oracle by at most the Newton error
# left at that mismatch.  The agreement bar is |dV| <= 1e-6 pu.
TOL_V_FP64 = 1e-9
TOL_V_MIXED = 1e-6
