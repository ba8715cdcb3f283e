"""Shared test setup: import paths, the `gpu` marker and common fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_PARENT = os.path.join(ROOT, "forceconstants.jl_b200")
for p in (ROOT, PKG_PARENT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and libfcb200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    return O


@pytest.fixture(scope="session")
def fcb():
    import fcb200
    return fcb200


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch.device("cuda:0")


# Argon FCC parameters of the reference's tests (test/runtests.jl:111-114).
AR = dict(a=5.2468, sigma=3.4, eps=0.24037, r_cut=8.5, mass=39.95)


def fcc_system(cells, std=0.0, seed=0):
    import fcb200
    sys_ = fcb200.FCC(AR["a"], "Ar", cells)
    if std > 0:
        sys_ = fcb200.displaced(sys_, std, seed)
    return sys_
