"""The Stillinger-Weber oracle is pinned to the reference's own derivative kernels.

Golden fixtures (tests/golden/sw_diamond_*.npz) were produced by the reference's
generated SW derivative kernels (translated from the reference checkout, see
tests/golden/make_sw_golden.py) driven by the restated triplet loop.  The
oracle's blocks come from exact hyper-dual arithmetic instead.
"""
import glob
import os

import numpy as np
import pytest

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sw_diamond_*.npz")))


def _dense(d):
    n = int(d["n"])
    flat = np.zeros(n ** 3)
    flat[d["ifc3_index"]] = d["ifc3_value"]
    return flat.reshape((n, n, n), order="F")


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
def test_oracle_matches_reference_kernels_golden(oracle, path):
    d = np.load(path)
    rc = float(d["r_cut"])
    psi = oracle.third_order_sw(d["positions"], d["box"], rc, float(d["tol"]))
    ref = _dense(d)
    assert np.max(np.abs(psi - ref)) <= 1e-12
    ifc2 = oracle.second_order_sw(d["positions"], d["box"], rc, float(d["tol"]))
    assert np.max(np.abs(ifc2 - d["ifc2"])) <= 1e-12


def test_cos0_per_family_is_required(oracle):
    """Using the truncated cosθ₀ for the iik block too breaks the 1e-12 parity."""
    d = np.load(GOLD[-1])
    rc = float(d["r_cut"])
    bad = oracle.third_order_sw(d["positions"], d["box"], rc, 1e-12, cos0_iik=oracle.COS0_GEN)
    assert np.max(np.abs(bad - _dense(d))) > 1e-12


def test_blocks_vs_translated_reference(oracle):
    if oracle.ref_lib() is None:
        pytest.skip("oracle/_ref/libswref.so not built (needs the reference checkout)")
    rng = np.random.default_rng(0)
    for _ in range(50):
        ri = rng.normal(size=3) * 3
        u = rng.normal(size=3)
        u *= rng.uniform(2.0, 3.7) / np.linalg.norm(u)
        v = rng.normal(size=3)
        v *= rng.uniform(2.0, 3.7) / np.linalg.norm(v)
        r9 = np.concatenate([ri, ri - u, ri - v])
        a, b = oracle.sw_blocks(r9), oracle.sw_blocks(r9, use_ref=True)
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b)))
        pa, pb = oracle.sw_pair_block(u), oracle.sw_pair_block(u, use_ref=True)
        assert np.max(np.abs(pa - pb)) <= 1e-12 * max(1.0, np.max(np.abs(pb)))


def test_sw_cutoff_assertion(oracle):
    d = np.load(GOLD[0])
    with pytest.raises(ValueError):
        oracle.third_order_sw(d["positions"], d["box"], 4.0, 1e-12)
