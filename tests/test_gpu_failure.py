"""The bounded-wait failure path of the tensor-core mode products.

Every mbarrier wait in the tcgen05 kernels is bounded; fcb200_set_wait_limit
sets the limit of the ordinary waits (default 2 s).  With a limit of 1 ns
the first wait that does not succeed at once gives up: the kernel records a
status word, drains the loads and MMAs it issued (the drains keep a 2 s
limit), frees its tensor memory and returns.  No trap, no fault: the host
reads FCB_ERR_TIMEOUT from fcb200_synchronize, and the same handle then runs a
normal call whose result matches the oracle — which it could not if tensor
memory had been left allocated (the next tcgen05.alloc would never succeed).
"""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu


def _err(k, ref):
    return float(np.max(np.abs(np.asarray(k, dtype=np.float64) - ref)) / np.max(np.abs(ref)))


def test_wait_limit_reports_timeout_and_handle_recovers(fcb, oracle, cuda_device):
    import torch
    from fcb200 import _lib
    L = _lib.lib()
    s = fcc_system((3, 3, 3), 0.05, 66)                     # n = 324: 411 tiles of 256 rows
    psi = oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    psi = oracle.mass_weight_third_order(psi, s.masses).astype(np.float32, order="F")
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    phi = np.asfortranarray(phi.astype(np.float32))
    ref = oracle.mcc3(psi.astype(np.float64), phi.astype(np.float64))
    d_psi, d_phi = torch.from_numpy(psi).to(cuda_device), torch.from_numpy(phi).to(cuda_device)
    h = _lib.handle(0)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(L.fcb200_synchronize(h, stream))              # nothing pending before the test
    try:
        _lib.check(L.fcb200_set_wait_limit(h, 1))
        fcb.mcc3(d_psi, d_phi, precision="bf16x3")           # device buffers: returns without a host wait
        st = L.fcb200_synchronize(h, stream)
    finally:
        _lib.check(L.fcb200_set_wait_limit(h, 0))            # back to the default limit
    assert st == _lib.FCB_ERR_TIMEOUT, (st, _lib.last_error())
    assert "bounded device-side wait" in _lib.last_error()[1]
    assert L.fcb200_synchronize(h, stream) == _lib.FCB_OK   # the status word was cleared
    for precision in ("bf16x3", "tf32x3"):
        k = fcb.mcc3(d_psi, d_phi, precision=precision)
        assert L.fcb200_synchronize(h, stream) == _lib.FCB_OK
        assert _err(k.cpu().numpy(), ref) <= 1e-5, precision
