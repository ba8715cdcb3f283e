"""Batched snapshots (fcb200_batch_*): every K3 of an eager run and of the
CUDA-graph replays equals the single-snapshot path bit for bit (the same
kernels and tiles: block-sparse first product and symmetric tiles for the
split precisions, dense FP32 products otherwise), also after positions change
between replays."""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu


def _phi(oracle, s):
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    return np.asfortranarray(phi.astype(np.float32))


@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_batch_matches_single_snapshots(fcb, oracle, cuda_device, precision):
    import torch
    from fcb200.batch import SnapshotBatch
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    cells = [(2, 2, 2), (3, 3, 3), (2, 2, 2), (3, 3, 2), (2, 2, 3)]
    systems = [fcc_system(c, 0.03 + 0.01 * i, 100 + i) for i, c in enumerate(cells)]
    phis = [_phi(oracle, s) for s in systems]
    b = SnapshotBatch(precision)
    outs = [b.add(s, pot, calc, p) for s, p in zip(systems, phis)]

    def single(s, p):
        _, k = fcb.snapshot_lj(s, pot, calc, torch.from_numpy(p).cuda(), precision=precision)
        torch.cuda.synchronize()
        return k.cpu().numpy()

    ref = [single(s, p) for s, p in zip(systems, phis)]
    b.run()                 # eager
    torch.cuda.synchronize()
    for o, r in zip(outs, ref):
        assert np.array_equal(o.cpu().numpy(), r)
    for o in outs:
        o.zero_()
    b.run()                 # captured and replayed as one graph
    b.run()
    torch.cuda.synchronize()
    info = b.info()
    # fp32: pair, self, dense writer, 3 mode products; split: pair, self,
    # neighbour-list memset + kernel, coefficients, phi split, sparse P1, P2, P3
    per_snapshot = 6 if precision == "fp32" else 9
    assert info["snapshots"] == len(systems) and info["lanes"] >= 1
    assert info["graph_nodes"] >= per_snapshot * len(systems)
    for o, r in zip(outs, ref):
        assert np.array_equal(o.cpu().numpy(), r)
    # new positions for snapshot 1, same graph
    moved = fcb.displaced(systems[1], 0.02, 7)
    b.set_positions(1, moved.positions)
    b.run()
    torch.cuda.synchronize()
    assert np.array_equal(outs[1].cpu().numpy(), single(moved, phis[1]))
    b.close()


def test_trajectory_k3_matches_single_snapshots(fcb, oracle, cuda_device, tmp_path):
    """An xyz trajectory (io.jl:319-353's frames) through trajectory_k3 in
    groups of two frames: every frame's K3 equals fcb200_snapshot_lj on the
    same positions bit for bit, the last group holding one frame only."""
    import torch
    from fcb200.batch import trajectory_k3
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    base = fcc_system((3, 3, 3))
    frames = [fcb.displaced(base, 0.03, 200 + t) for t in range(5)]
    path = tmp_path / "traj.xyz"
    with open(path, "w") as f:
        for t, s in enumerate(frames):
            f.write(f"{s.n_atoms}\nTimestep: {t}\n")
            f.write("".join(f"{i + 1} {x!r} {y!r} {z!r}\n" for i, (x, y, z) in enumerate(s.positions.tolist())))
    phi = _phi(oracle, base)                      # modes of the perfect lattice, shared by every frame
    seen = []
    got = trajectory_k3(str(path), base.n_atoms, 6, base.box_sizes, base.masses, pot, calc, phi,
                        frames_per_batch=2)
    trajectory_k3(str(path), base.n_atoms, 6, base.box_sizes, base.masses, pot, calc, phi, frames_per_batch=2,
                  on_frame=lambda t, ids, k3: seen.append((t, ids.tolist(), k3.cpu().numpy())))
    assert len(got) == 5 and [t for t, _, _ in seen] == [0, 1, 2, 3, 4]   # the sixth frame is not in the file
    d_phi = torch.from_numpy(phi).to(cuda_device)
    for s, k, (_, ids, k2) in zip(frames, got, seen):
        _, ref = fcb.snapshot_lj(s, pot, calc, d_phi, precision="bf16x3")
        torch.cuda.synchronize()
        ref = ref.cpu().numpy()
        assert ids == list(range(1, s.n_atoms + 1))
        assert np.array_equal(k, ref) and np.array_equal(k2, ref)


def test_batch_admission_refuses_oversize(fcb, cuda_device):
    from fcb200 import _lib
    from fcb200.batch import SnapshotBatch
    s = fcc_system((2, 2, 2), 0.03, 1)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    b = SnapshotBatch("bf16x3", hbm_budget_bytes=1 << 20)   # 1 MiB of scratch: too small
    b.add(s, pot, calc, np.eye(96, dtype=np.float32))
    with pytest.raises(_lib.FCB200Error) as e:
        b.run()
    assert e.value.code == _lib.FCB_ERR_OOM
    b.close()


def test_autotune_cache_roundtrip(fcb, cuda_device, tmp_path):
    from fcb200.batch import autotune_mcc3
    path = str(tmp_path / "tune.json")
    autotune_mcc3(96, "bf16x3", path)
    text = open(path).read()
    assert "mode_tiles" in text
    autotune_mcc3(96, "bf16x3", path)     # cached: no retune, file stays valid
    assert "mode_tiles" in open(path).read()


def test_batch_replans_when_neighbourhoods_grow(fcb, oracle, cuda_device):
    """Positions compressed by 8 % bring more atoms inside the cutoff than the
    sparse tables were sized for when the snapshot was added; set_positions
    re-plans the batch, and the result still equals the single-snapshot path."""
    import torch
    from fcb200.batch import SnapshotBatch
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    s = fcc_system((4, 4, 4), 0.03, 41)
    phi = _phi(oracle, s)
    b = SnapshotBatch("bf16x3")
    out = b.add(s, pot, calc, phi)
    b.run()
    b.run()
    b.run()
    squeezed = fcb.SuperCellSystem(s.positions * 0.92, s.masses, s.box_sizes)
    b.set_positions(0, squeezed.positions)
    b.run()
    torch.cuda.synchronize()
    _, k = fcb.snapshot_lj(squeezed, pot, calc, torch.from_numpy(phi).cuda(), precision="bf16x3")
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), k.cpu().numpy())
    b.close()
