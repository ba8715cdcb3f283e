"""The finite-difference oracle (oracle/fd_oracle.c, restating
src/finitediff/*.jl) against the analytical oracle, which the golden values
pin: FD third-order elements and FD IFC2 agree with the analytical LJ force
constants within the O(h²) truncation of the reference's default step.  CPU
only."""
import numpy as np

from conftest import AR, atoms_clear_of_cutoff, fcc_system

H = 0.04 * 0.5291772109


def test_fd_oracle_third_order_lj(oracle):
    s = fcc_system((4, 4, 4), 0.05, 77)
    psi = oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 0.0)
    a, b, c = (int(x) for x in atoms_clear_of_cutoff(s, AR["r_cut"])[:3])
    el = np.array([[a, 0, b, 1, a, 0], [a, 2, a, 2, a, 2], [b, 1, c, 0, b, 1], [a, 0, b, 1, c, 2],
                   [a, 0, a, 1, b, 1]], dtype=np.int64)
    fd = oracle.fd_third_order("lj", s.positions, s.box_sizes, el, H, AR["sigma"], AR["eps"], AR["r_cut"])
    want = [psi[3 * a, 3 * b + 1, 3 * a], psi[3 * a + 2, 3 * a + 2, 3 * a + 2], psi[3 * b + 1, 3 * c, 3 * b + 1],
            psi[3 * a, 3 * b + 1, 3 * c + 2]]
    assert np.max(np.abs(fd[:4] - want)) <= 2e-3 * np.max(np.abs(psi))
    assert np.isnan(fd[4])                   # i == j != k: no stencil in the reference


def test_fd_oracle_second_order_lj(oracle):
    s = fcc_system((2, 2, 2), 0.04, 8)
    fd = oracle.fd_second_order("lj", s.positions, s.box_sizes, 4.5, H, AR["sigma"], AR["eps"], 4.5)
    ana = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], 4.5, 0.0)
    assert np.max(np.abs(fd - ana)) <= 2e-3 * np.max(np.abs(ana))
