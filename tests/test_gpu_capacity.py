"""The fixed neighbour capacity of the block-sparse snapshot path
(fcb200_set_neighbour_capacity).

By default fcb200_snapshot_lj reads the largest neighbour count back to the
host once per call.  With a capacity fixed on the handle it does not, so:

* the FP64 Ψ and K3 equal those of the default path bit for bit (the tables
  only gain zero rows: 96 slots per atom against the default's 80 on the
  256-atom cell);
* the call can be captured in a CUDA graph, after one uncaptured call has
  sized the handle's scratch, and every replay rewrites the same K3;
* a capacity below the largest neighbourhood (8 slots against 79 neighbours
  with the atom itself) is reported as FCB_ERR_ARG (by the call itself, which
  synchronises when its positions are on the host), and the handle then runs a
  normal call again.
"""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cell(fcb, oracle):
    s = fcc_system((4, 4, 4), 0.05, 1234)
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    return s, np.asfortranarray(phi.astype(np.float32))


def _run(fcb, s, d_phi, psi, k3, stream=0):
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    fcb.snapshot_lj(s, pot, calc, d_phi, precision="bf16x3", psi_out=psi, k3_out=k3, stream=stream)


def test_fixed_capacity_matches_default_and_captures(fcb, cuda_device, cell):
    import torch
    from fcb200.arrays import julia_empty
    s, phi = cell
    n = 3 * s.n_atoms
    d_phi = torch.from_numpy(phi).to(cuda_device)
    d_pos = torch.from_numpy(s.positions).to(cuda_device)
    d_box = torch.from_numpy(s.box_sizes).to(cuda_device)
    d_m = torch.from_numpy(s.masses).to(cuda_device)
    psi = julia_empty((n, n, n), np.float64, "cuda")
    k3 = julia_empty((n, n, n), np.float32, "cuda")
    _run(fcb, s, d_phi, psi, k3)
    torch.cuda.synchronize()
    psi_ref, k3_ref = psi.clone(), k3.clone()
    try:
        fcb.set_neighbour_capacity(96)
        psi.fill_(np.nan)
        k3.fill_(np.nan)
        _run(fcb, s, d_phi, psi, k3)
        torch.cuda.synchronize()
        assert torch.equal(psi, psi_ref) and torch.equal(k3, k3_ref)

        # device-resident positions, box and masses: nothing crosses to the host
        from fcb200 import _lib
        from fcb200.arrays import ptr
        L, h = _lib.lib(), _lib.handle(0)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())

        def call(stream):
            _lib.check(L.fcb200_snapshot_lj(h, ptr(d_pos), s.n_atoms, ptr(d_box), float(AR["sigma"]),
                                            float(AR["eps"]), float(AR["r_cut"]), 1e-12, ptr(d_m), ptr(d_phi), 0,
                                            n, _lib.PRECISIONS["bf16x3"], ptr(psi), ptr(k3), stream))

        with torch.cuda.stream(side):
            call(side.cuda_stream)                     # sizes the scratch outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side, capture_error_mode="relaxed"):
            call(side.cuda_stream)
        psi.fill_(np.nan)
        k3.fill_(np.nan)
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(psi, psi_ref) and torch.equal(k3, k3_ref)
        _lib.check(L.fcb200_synchronize(h, 0))
        del g
    finally:
        fcb.set_neighbour_capacity(0)


def test_capacity_overflow_reported_and_handle_recovers(fcb, cuda_device, cell):
    import torch
    from fcb200 import _lib
    from fcb200.arrays import julia_empty
    s, phi = cell
    n = 3 * s.n_atoms
    d_phi = torch.from_numpy(phi).to(cuda_device)
    psi = julia_empty((n, n, n), np.float64, "cuda")
    k3 = julia_empty((n, n, n), np.float32, "cuda")
    L, h = _lib.lib(), _lib.handle(0)
    _run(fcb, s, d_phi, psi, k3)
    _lib.check(L.fcb200_synchronize(h, 0))
    k3_ref = k3.clone()
    try:
        fcb.set_neighbour_capacity(8)
        with pytest.raises(_lib.FCB200Error) as e:
            _run(fcb, s, d_phi, psi, k3)         # host positions: the call synchronises and reports
            _lib.check(L.fcb200_synchronize(h, 0))
        assert e.value.code == _lib.FCB_ERR_ARG
    finally:
        fcb.set_neighbour_capacity(0)
    k3.fill_(np.nan)
    _run(fcb, s, d_phi, psi, k3)
    _lib.check(L.fcb200_synchronize(h, 0))
    assert torch.equal(k3, k3_ref)
    with pytest.raises(_lib.FCB200Error):
        fcb.set_neighbour_capacity(-1)
