"""The allocation-free LJ assembly entry point, called through the C ABI.

fcb200_third_order_lj_noalloc exists for callers that cannot let a library
allocate device memory (a Julia host whose device memory belongs to CUDA.jl's
pool, programs that size all device memory at start-up, callers that cannot
afford the device-wide synchronisation of cudaFree).  Its scratch is a fixed
device array shared by every call, so this test checks it against the regular
entry point (fcb200_third_order_lj, bit-exact as all assembly tests here) on
two different systems in a row: the second call must not be affected by what
the first one left in the shared array.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one.  A further test queues two calls on one
non-default stream with no host synchronisation between them.
"""
import ctypes

import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu


def _regular(fcb, s, masses, flags, weighted_out32):
    import torch
    from fcb200 import _lib
    from fcb200.arrays import julia_empty
    n = 3 * s.n_atoms
    psi = julia_empty((n, n, n), np.float64, "cuda")
    psi32 = julia_empty((n, n, n), np.float32, "cuda") if weighted_out32 else None
    m = torch.from_numpy(masses).cuda()
    _lib.check(_lib.lib().fcb200_third_order_lj(
        _lib.handle(0), s.positions.ctypes.data, s.n_atoms, s.box_sizes.ctypes.data, AR["sigma"], AR["eps"],
        AR["r_cut"], 1e-12, int(m.data_ptr()), int(psi.data_ptr()),
        int(psi32.data_ptr()) if psi32 is not None else None, flags, None))
    torch.cuda.synchronize()
    return psi.cpu().numpy(), (psi32.cpu().numpy() if psi32 is not None else None)


def _noalloc(fcb, s, masses, flags, weighted_out32):
    import torch
    from fcb200 import _lib
    from fcb200.arrays import julia_empty
    n = 3 * s.n_atoms
    pos = torch.from_numpy(s.positions).cuda()
    m = torch.from_numpy(masses).cuda()
    psi = julia_empty((n, n, n), np.float64, "cuda")
    psi32 = julia_empty((n, n, n), np.float32, "cuda") if weighted_out32 else None
    psi.fill_(np.nan)
    box = np.ascontiguousarray(s.box_sizes)
    st = _lib.lib().fcb200_third_order_lj_noalloc(
        int(pos.data_ptr()), s.n_atoms, box.ctypes.data, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12,
        int(m.data_ptr()), int(psi.data_ptr()), int(psi32.data_ptr()) if psi32 is not None else None, flags,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)
    torch.cuda.synchronize()
    return psi.cpu().numpy(), (psi32.cpu().numpy() if psi32 is not None else None)


def test_noalloc_matches_regular_entry_point_twice(fcb, cuda_device):
    from fcb200 import _lib
    # First call: 256 atoms (the maximum), unweighted Ψ plus the FP32 mass-weighted copy.
    s1 = fcc_system((4, 4, 4), 0.05, 101)
    m1 = np.linspace(35.0, 45.0, s1.n_atoms)
    a64, a32 = _noalloc(fcb, s1, m1, 0, True)
    r64, r32 = _regular(fcb, s1, m1, 0, True)
    assert np.array_equal(a64, r64)
    assert np.array_equal(a32, r32)
    # Second call right after: a smaller, different system, mass-weighted FP64.
    s2 = fcc_system((3, 3, 3), 0.08, 202)
    m2 = np.full(s2.n_atoms, 39.95)
    b64, _ = _noalloc(fcb, s2, m2, _lib.FCB_PSI_MASS_WEIGHTED, False)
    q64, _ = _regular(fcb, s2, m2, _lib.FCB_PSI_MASS_WEIGHTED, False)
    assert np.array_equal(b64, q64)


def test_noalloc_rejects_oversize_and_host_buffers(fcb, cuda_device):
    import torch
    from fcb200 import _lib
    L = _lib.lib()
    big = fcc_system((4, 4, 5))                     # 320 atoms > FCB_NOALLOC_MAX_ATOMS
    pos = torch.from_numpy(big.positions).cuda()
    out = torch.empty(8, dtype=torch.float64, device="cuda")
    box = np.ascontiguousarray(big.box_sizes)
    st = L.fcb200_third_order_lj_noalloc(int(pos.data_ptr()), big.n_atoms, box.ctypes.data, AR["sigma"],
                                         AR["eps"], AR["r_cut"], 1e-12, None, int(out.data_ptr()), None, 0, None)
    assert st == _lib.FCB_ERR_ARG
    assert "exceeds the fixed scratch" in _lib.last_error()[1]
    small = fcc_system((2, 2, 2))
    host_out = np.zeros(96 ** 3)
    st = L.fcb200_third_order_lj_noalloc(small.positions.ctypes.data, small.n_atoms,
                                         np.ascontiguousarray(small.box_sizes).ctypes.data, AR["sigma"], AR["eps"],
                                         AR["r_cut"], 1e-12, None, host_out.ctypes.data, None, 0, None)
    assert st == _lib.FCB_ERR_ARG
    assert "device memory" in _lib.last_error()[1]


def test_noalloc_back_to_back_on_one_stream(fcb, cuda_device):
    """Two calls of different sizes queued on one non-default stream with no
    host synchronisation between them — the way the shared scratch is meant to
    be used, since calls on one stream run one after the other — and a single
    synchronisation at the end: both results equal the regular entry point."""
    import torch
    from fcb200 import _lib
    from fcb200.arrays import julia_empty
    L = _lib.lib()
    s1, s2 = fcc_system((4, 4, 4), 0.04, 303), fcc_system((3, 3, 3), 0.06, 404)
    m1, m2 = np.full(s1.n_atoms, 39.95), np.linspace(30.0, 50.0, s2.n_atoms)
    stream = torch.cuda.Stream()
    outs = []
    with torch.cuda.stream(stream):
        for s, m in ((s1, m1), (s2, m2)):
            n = 3 * s.n_atoms
            pos = torch.from_numpy(s.positions).cuda()
            dm = torch.from_numpy(m).cuda()
            psi = julia_empty((n, n, n), np.float64, "cuda")
            psi32 = julia_empty((n, n, n), np.float32, "cuda")
            box = np.ascontiguousarray(s.box_sizes)
            _lib.check(L.fcb200_third_order_lj_noalloc(
                int(pos.data_ptr()), s.n_atoms, box.ctypes.data, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12,
                int(dm.data_ptr()), int(psi.data_ptr()), int(psi32.data_ptr()), 0,
                ctypes.c_void_p(stream.cuda_stream)))
            outs.append((pos, dm, psi, psi32))
    stream.synchronize()
    for (s, m), (_, _, psi, psi32) in zip(((s1, m1), (s2, m2)), outs):
        r64, r32 = _regular(fcb, s, m, 0, True)
        assert np.array_equal(psi.cpu().numpy(), r64)
        assert np.array_equal(psi32.cpu().numpy(), r32)
