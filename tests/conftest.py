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


def atoms_clear_of_cutoff(sys_, r_cut, margin=0.05):
    """Atoms with no pair distance (single minimum image) within `margin` of
    r_cut (the stencils move a pair by at most 2h = 0.042 Å).  A truncated (unshifted) pair energy jumps at r_cut, so a
    finite-difference stencil that moves such a pair across it measures the
    jump, in the reference as in any restatement of it."""
    p = np.asarray(sys_.positions).reshape(-1, 3)
    d = p[:, None, :] - p[None, :, :]
    d -= sys_.box_sizes * np.round(d / sys_.box_sizes)
    dist = np.linalg.norm(d, axis=2)
    near = (np.abs(dist - r_cut) < margin) & (dist > 0)
    return np.nonzero(~near.any(axis=1))[0]
