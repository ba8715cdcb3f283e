"""Benchmark: one LJ snapshot through IFC3 assembly + mcc3 per step.

Workload (the precision configuration): 256-atom FCC argon (4×4×4 cells,
a = 5.2468 Å), positions displaced by i.i.d. N(0, 0.05²) Å (seeded),
σ = 3.4 Å, ϵ = 0.24037 kcal/mol, r_cut = 8.5 Å, tol = 1e-12, m = 39.95 u;
φ = eigenvectors of the dynamical matrix (FP32).  One step = dense FP64 IFC3
assembly (+ASR, tol) with the fused mass-weighted split operand, then mcc3 over
all 768 modes (three mode products), K3 in FP32.  Inputs are synthetic (seeded).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision bf16x3|tf32x3|fp32]
                    [--impl ours|reference] [--out-dir DIR]

Prints one JSON line (rank 0).  Time-like metric: value = seconds per snapshot
for the whole job (max over ranks of the device time ÷ all snapshots).  N > 1
runs N independent replicas (one snapshot stream per GPU, no collective on the
data path).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "forceconstants.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "IFC3+mcc3 s/snapshot (256-atom LJ), split-BF16 vs FP32 GPU at ≤1e-5 rel err"
UNIT = "s/snapshot"
CELLS, A_LAT, STD, SEED = (4, 4, 4), 5.2468, 0.05, 1234
SIGMA, EPS, R_CUT, TOL, MASS = 3.4, 0.24037, 8.5, 1e-12, 39.95
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
# DRAM bytes (read + write) per launch at n = 768, bf16x3, from one 1-pass ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) of
#   python bench.py --steps 2 --warmup 3 --skip-cpu --skip-e2e --skip-batch --skip-extra
# (profiles/launch_list_snapshot_lj_256atoms_bf16x3.md): the compact form's
# grouped second product 0.759e9 + 1.157e9, its MN-major third product
# 1.541e9 + 1.764e9, the FP64 writer 0.005e9 + 3.561e9; the dense-layout
# symmetric product (taken where the compact form does not pay) 3.770e9.
NCU_TRAFFIC = {"mode_product_tc2_p2": 1.914e9, "mode_product_tc2_p3": 3.138e9, "mode_product_tc2_sym": 3.770e9,
               "ifc3_dense_psi64": 3.566e9}


def sym_executed_flops(R, F, K, M, split=3):
    """Tensor flops one symmetric pair-kernel launch executes: 256-row tiles ×
    mode tiles of width bn (default tiling: ceil(M/256) tiles), a tile live when
    its last column reaches its first row's outer index r // F."""
    n_tiles = -(-M // 256)
    bn = -(-(-(-M // n_tiles)) // 16) * 16
    kpad = -(-K // 64) * 64
    live = 0
    for mt in range(-(-R // 256)):
        pmin = (mt * 256) // F
        for nt in range(n_tiles):
            if min(nt * bn + bn, M) - 1 >= pmin:
                live += 1
    return 2.0 * 256 * bn * kpad * live * split


def full_sym_executed_flops(Mp, M, K, split=3, packed=False):
    """Tensor flops of the third product with full symmetry: 256-row tiles
    (rows a + Mp·b) computed when a // 256 <= b // 256, each over every 256-wide
    mode tile (with the packed output: a0 <= b and only the mode tiles that
    reach s >= b), K padded to whole 64-wide chunks."""
    n_tiles = -(-M // 256)
    bn = 256 if M > 256 else -(-M // 16) * 16
    kpad = -(-K // 64) * 64
    live = 0
    for mt in range(Mp * M // 256):
        a0, b = (mt * 256) % Mp, (mt * 256) // Mp
        if packed:
            live += sum(1 for nt in range(n_tiles) if a0 <= b and min(nt * bn + bn, M) - 1 >= b)
        elif a0 // 256 <= b // 256:
            live += n_tiles
    return 2.0 * 256 * bn * kpad * live * split


def sparse_cap(pos, box, r_cut):
    """Capacity of the sparse coefficient tables, as the library sizes them for a
    single snapshot: the largest neighbourhood (atoms within r_cut by the single
    minimum image, the atom itself included), rounded up to a multiple of 4."""
    p = np.asarray(pos).reshape(-1, 3)
    d = p[:, None, :] - p[None, :, :]
    d -= box * np.round(d / box)
    cnt = int(((d * d).sum(-1) < r_cut * r_cut).sum(1).max())
    return -(-cnt // 4) * 4


def compact_shapes(n, M, cap):
    """(Mp, Kc) of the compact sparse products when the library takes that form
    (modes padded to 256-row blocks, neighbourhood rows to 8; taken when it
    executes at least 10 % fewer tile flops than the dense-K pair), else None."""
    if M % 8:
        return None
    Mp, Kc = -(-M // 256) * 256, -(-3 * cap // 8) * 8
    return (Mp, Kc) if Mp * n * Kc + Mp * M * n < 0.9 * (n * M * n + M * M * n) else None


def inner_sym_executed_flops(n, M, Mp, Kc, split=3):
    """Tensor flops of the grouped second product: per column k, 256 × 256 tiles
    (p, q) with q-tile >= p-tile, K padded to whole 64-wide chunks."""
    q_tiles = -(-M // 256)
    live = sum(1 for pt in range(Mp // 256) for qt in range(q_tiles) if min(qt * 256 + 256, M) - 1 >= pt * 256)
    return 2.0 * 256 * 256 * (-(-Kc // 64) * 64) * live * n * split


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return FALLBACK_PEAKS, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks / throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, out_dir: str):
        self.idx = gpu_index
        self.proc = None
        self.path = os.path.join(out_dir, f"clocks_bench_{os.getpid()}.csv")
        self.nvml = None
        self.samples = []

    def _nvml_handle(self):
        """NVML handle of the CUDA device `idx` (matched by PCI bus id, so that a
        CUDA_VISIBLE_DEVICES mapping does not pick another GPU)."""
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.idx)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.idx)

    def _sample(self):
        nv, h = self.nvml
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((sm, [k for k, b in bits.items() if r & b]))

    def _poll(self):
        while not self.halt.is_set():
            try:
                self._sample()
            except Exception:
                return
            time.sleep(0.002)

    def wait_for(self, event):
        """Samples from the calling thread until `event` (recorded after the
        timed steps) has completed, so that the timed region is sampled even
        when the background thread gets little time."""
        while not event.query():
            if self.nvml is not None:
                try:
                    self._sample()
                except Exception:
                    pass
            time.sleep(0.0005)

    def start(self):
        """nvidia-smi writes its CSV record (100 ms period) and an NVML thread
        samples the SM clock and the throttle reasons every 2 ms, so that a
        timed region of a few tens of milliseconds still holds samples."""
        import threading
        try:
            self.nvml = self._nvml_handle()
            self.smax = self.nvml[0].nvmlDeviceGetMaxClockInfo(self.nvml[1], self.nvml[0].NVML_CLOCK_SM)
            self.halt = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception:
            self.nvml = None
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        nvml = None
        if self.nvml is not None:
            self.halt.set()
            self.thread.join(timeout=5)
            if self.samples:
                nvml = {"sm_mhz": statistics.median(x[0] for x in self.samples), "sm_max_mhz": float(self.smax),
                        "reasons": sorted({r for x in self.samples for r in x[1]}), "samples": len(self.samples),
                        "source": "NVML, timed region only (polled while the timed steps run)"}
        if self.proc is None:
            return nvml or {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        smi = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
               "reasons": sorted(reasons), "samples": len(sm)}
        if nvml is None:
            return smi
        nvml["nvidia_smi"] = smi  # 100 ms record, including the 0.25 s after the timed region
        return nvml


def build_workload(fcb, device):
    import torch
    s = fcb.displaced(fcb.FCC(A_LAT, "Ar", CELLS), STD, SEED)
    pot = fcb.LJ(SIGMA, EPS, R_CUT)
    calc = fcb.AnalyticalCalculator(TOL, R_CUT)
    dyn = fcb.dynamical_matrix(s, pot, calc)               # on the GPU (fcb200_second_order_lj)
    _, phi = fcb.get_modes(dyn)                             # on the GPU (fcb200_get_modes, cuSOLVER syevd)
    phi32 = np.asfortranarray(phi.astype(np.float32))
    return s, pot, calc, phi32


def julia_tensor(shape, dtype, device):
    from fcb200.arrays import julia_empty
    return julia_empty(shape, dtype, device)


def fp64_reference_k3(psi64_dev, masses, phi32):
    """FP64 K3 of the same inputs on the GPU (torch float64 tensordot), used
    only to report the error of the timed path; not part of the timed region."""
    import torch
    n = psi64_dev.shape[0]
    m = torch.from_numpy(np.repeat(masses, 3)).cuda()
    w = torch.rsqrt(m[:, None, None] * m[None, :, None] * m[None, None, :])
    mw = (psi64_dev * w).contiguous()                       # [i,j,k] semantics preserved
    phi = torch.from_numpy(np.ascontiguousarray(phi32.astype(np.float64))).cuda()
    k1 = torch.tensordot(phi, mw, dims=([0], [0]))          # [n, j, k]
    del mw
    k2 = torch.tensordot(k1, phi, dims=([1], [0]))          # [n, k, m]
    del k1
    k3 = torch.tensordot(k2, phi, dims=([1], [0]))          # [n, m, l]
    return k3


def err_vs(k3_dev, ref):
    import torch
    d = k3_dev.to(torch.float64) - ref
    scale = ref.abs().max()
    return {"max_rel": float(d.abs().max() / scale),
            "rms_rel": float(torch.sqrt((d * d).mean()) / torch.sqrt((ref * ref).mean()))}


def cpu_baseline(phi32, threads=None):
    """The oracle (CPU restatement of the reference path) on the host cores, one
    whole snapshot measured: 256-atom third_order (all threads), serial mass
    weighting, the FP32 cast, and the FP64 mcc3 over all 768 modes (three mode
    products, numpy BLAS on all threads) with the same φ as the GPU step."""
    from oracle import oracle as O
    import fcb200 as fcb
    if threads:
        O.set_threads(threads)
    s = fcb.displaced(fcb.FCC(A_LAT, "Ar", CELLS), STD, SEED)
    n = 3 * s.n_atoms
    t0 = time.perf_counter()
    psi = O.third_order_lj(s.positions, s.box_sizes, SIGMA, EPS, R_CUT, TOL)
    t1 = time.perf_counter()
    O.mass_weight_third_order(psi, s.masses)
    t2 = time.perf_counter()
    f32 = np.empty(n ** 3, np.float32)
    O.lib().oracle_cast_f32(O._pd(psi.reshape(-1, order="F")), f32.ctypes.data_as(O._PF), n ** 3)
    t3 = time.perf_counter()
    del psi
    psi32 = f32.reshape((n, n, n), order="F")
    t4 = time.perf_counter()
    _ = O.mcc3(psi32, phi32)
    t5 = time.perf_counter()
    total = t5 - t0 - (t4 - t3)
    return {"value": total, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": (f"one whole 256-atom snapshot by the oracle, all measured: third_order {t1 - t0:.2f}s "
                       f"({O.num_threads()} threads) + serial mass_weight {t2 - t1:.2f}s + cast {t3 - t2:.2f}s + "
                       f"FP64 mcc3 over 768 modes {t5 - t4:.2f}s (numpy BLAS)")}


def batch_config(fcb, precision, device, out_dir, reps=3):
    """The batching configuration: 48 LJ argon snapshots of uneven size (16 each
    of FCC 3x3x3 = 108, 4x4x4 = 256 and 5x5x4 = 400 atoms), displacement std
    drawn from U(0.03, 0.08) A per snapshot (seeded), through assembly, mass
    weighting and full-mode mcc3 as one CUDA-graph launch per batch.  phi per
    size class from the perfect lattice (the modes of the reference structure,
    shared by its snapshots).  The scratch budget admits two lanes; every lane
    has its own K3 buffer per size class (snapshots of one lane run one after
    another, fcb200_batch_lane), and after the timed runs the last K3 of each
    size class is checked bit for bit against the single-snapshot path."""
    import torch
    from fcb200.batch import SnapshotBatch, autotune_mcc3
    rng = np.random.default_rng(4242)
    pot = fcb.LJ(SIGMA, EPS, R_CUT)
    calc = fcb.AnalyticalCalculator(TOL, R_CUT)
    classes = [(3, 3, 3), (4, 4, 4), (5, 5, 4)]
    lanes = 2
    t0 = time.perf_counter()
    cache = os.path.join(out_dir, "autotune_mcc3.json")
    for c in classes:
        autotune_mcc3(12 * c[0] * c[1] * c[2], precision, cache)
    tune_s = time.perf_counter() - t0
    b = SnapshotBatch(precision, hbm_budget_bytes=int(1.2 * (2 * 2 * 1200 * (3 * 1200 ** 2 + 1200) + 40e6)))
    outs, members, phis = {}, [], {}
    for c in classes:
        base = fcb.FCC(A_LAT, "Ar", c)
        dyn = fcb.dynamical_matrix(base, pot, calc)
        _, phi = fcb.get_modes(dyn)
        phis[c] = np.asfortranarray(phi.astype(np.float32))
        n = 3 * base.n_atoms
        outs[c] = [julia_tensor((n, n, n), np.float32, device) for _ in range(lanes)]
        for j in range(16):
            s = fcb.displaced(base, float(rng.uniform(0.03, 0.08)), int(rng.integers(1 << 30)))
            b.add(s, pot, calc, phis[c], k3_out=outs[c][j % lanes])
            members.append((c, j % lanes, s))
    stream = torch.cuda.current_stream()
    sp = int(stream.cuda_stream)
    b.run(sp)                 # eager: makes the plan and sizes the lane scratch
    info = b.info()
    for i, (c, slot, _) in enumerate(members):
        if info["lanes"] != lanes or b.lane(i) != slot:
            raise RuntimeError("the batch plan does not put the snapshots that share a K3 buffer in one lane")
    b.run(sp)                 # capture + first graph launch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        b.run(sp)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    info = b.info()
    # the last snapshot of each size class in lane 0 wrote that class's lane-0 buffer last
    checked = {}
    for c in classes:
        last = [s for (cc, slot, s) in members if cc == c and slot == 0][-1]
        _, k = fcb.snapshot_lj(last, pot, calc, torch.from_numpy(phis[c]).to(device), precision=precision)
        torch.cuda.synchronize()
        checked[f"{3 * last.n_atoms}"] = bool(torch.equal(k, outs[c][0]))
    b.close()
    del outs
    torch.cuda.empty_cache()
    if not all(checked.values()):
        raise RuntimeError(f"batch K3 differs from the single-snapshot path: {checked}")
    return {"snapshots": info["snapshots"], "s_per_batch": ms / 1e3, "snapshots_per_s": info["snapshots"] / (ms / 1e3),
            "s_per_snapshot": ms / 1e3 / info["snapshots"], "graph_launches_per_batch": 1,
            "graph_nodes": info["graph_nodes"], "lanes": info["lanes"], "scratch_bytes": info["scratch_bytes"],
            "autotune_s": round(tune_s, 2), "precision": precision,
            "k3_buffers": "one per lane and size class (snapshots of a lane run in sequence)",
            "bitwise_equal_to_single_snapshot_path": checked,
            "workload": "48 LJ snapshots: 16x108, 16x256, 16x400 atoms, std U(0.03,0.08) A, full-mode mcc3"}


def gemm_peaks(device, reps=10):
    """Dense GEMM throughput of this GPU, the roofline denominators of the FP32
    and TF32x3 forms (MEASURED_PEAKS.json holds the HBM copy and BF16 GEMM
    figures only): torch.matmul (cuBLAS) of 8192 x 8192 FP32 matrices with
    TF32 off (FFMA) and on (tensor cores), CUDA events around `reps` calls
    after 3 warm-up calls (a burst, like MEASURED_PEAKS.json's bf16_tflops)."""
    import torch
    n = 8192
    a, b = torch.randn(n, n, device=device), torch.randn(n, n, device=device)
    c = torch.empty(n, n, device=device)
    prev = torch.backends.cuda.matmul.allow_tf32
    out = {}
    try:
        for name, tf32 in (("fp32_tflops", False), ("tf32_tflops", True)):
            torch.backends.cuda.matmul.allow_tf32 = tf32
            for _ in range(3):
                torch.matmul(a, b, out=c)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                torch.matmul(a, b, out=c)
            e1.record()
            torch.cuda.synchronize()
            out[name] = round(2.0 * n ** 3 * reps / (e0.elapsed_time(e1) * 1e-3) / 1e12, 1)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b, c
    torch.cuda.empty_cache()
    out["method"] = f"torch.matmul FP32 {n}^3, TF32 off / on, {reps} calls after 3 warm-up, CUDA events"
    return out


def timed(fn, stream, reps):
    """Mean device time (s) of fn() over `reps` calls, CUDA events on `stream`."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps / 1e3


def sw_snapshot_config(fcb, device, stream, reps=3):
    """The three-body configuration: Stillinger-Weber diamond Si 3x3x3 (216
    atoms, n = 648), displaced std 0.03 A (seed 216), φ from its dynamical
    matrix (on the GPU); one step = fcb200_snapshot_sw (FP64 SW IFC3 with ASR,
    the mass-weighted operand, mcc3 over all 648 modes)."""
    import torch
    s = fcb.displaced(fcb.Diamond(5.43, "Si", (3, 3, 3)), 0.03, 216)
    pot = fcb.StillingerWeberSilicon()
    calc = fcb.AutoDiffCalculator(TOL, pot.r_cut)
    dyn = fcb.dynamical_matrix(s, pot, calc, device=device)
    _, _, phi = fcb.get_modes(dyn, 3, phi32=True)
    n = 3 * s.n_atoms
    psi = julia_tensor((n, n, n), np.float64, device)
    k3 = julia_tensor((n, n, n), np.float32, device)
    sp = int(stream.cuda_stream)
    out = {"workload": "SW diamond Si 3x3x3 (216 atoms, n=648), std 0.03 A seed 216, all 648 modes, FP64 Psi written"}
    ref = None
    for precision in ("bf16x3", "tf32x3", "fp32"):
        def step():
            fcb.snapshot_lj(s, pot, calc, phi, precision=precision, psi_out=psi, k3_out=k3, stream=sp)
        step()
        torch.cuda.synchronize()
        if ref is None:
            ref = fp64_reference_k3(psi, s.masses, phi.cpu().numpy())
        out[precision] = {"s_per_snapshot": timed(step, stream, reps), "error_vs_fp64": err_vs(k3, ref)}
    del ref, psi, k3
    torch.cuda.empty_cache()
    return out


def adjoint_config(fcb, device, stream, s, pot, calc, reps=3):
    """The differentiation configuration: the 256-atom displaced cell, φ frozen,
    W ~ N(0,1) over the first 256 modes (seeded); one call of
    fcb200_mcc3_adjoint_lj gives dL/dpositions (768), dL/dsigma, dL/deps and L
    (device inputs; it synchronises once to read the scalars)."""
    import torch
    from fcb200.adjoint import mcc3_adjoint_lj
    from fcb200.arrays import as_julia
    M = 256
    dyn = fcb.dynamical_matrix(s, pot, calc, device=device)
    _, _, phi = fcb.get_modes(dyn, 3, phi32=True)
    W = as_julia(torch.from_numpy(np.random.default_rng(2025).normal(size=(M, M, M)).astype(np.float32)).to(device),
                 np.float32)
    out = {"workload": "256-atom LJ cell (std 0.05 A seed 1234), W over modes 0..255, grads of L = sum W*K3",
           "checked": "tests/test_gpu_adjoint.py: all 768 position components, sigma and eps within 1e-6 of "
                      "central differences (h = 1e-5 A) with G in FP64"}
    for precision in ("fp64", "tf32x3", "fp32"):
        def call():
            mcc3_adjoint_lj(s, pot, calc, phi, W, precision=precision)
        call()
        out[precision] = {"s_per_call": timed(call, stream, reps)}
    del W
    torch.cuda.empty_cache()
    return out


def config1(fcb, device, stream, reps=3):
    """The plain configuration: the perfect 256-atom lattice, FP64 IFC3 with the
    fused FP32 mass-weighted copy, φ = FP32 eigenvectors of the dynamical
    matrix (on the GPU), then FP32 mcc3 with block_size = 256 (27 blocks, the
    result in host memory as mcc.jl:89-120 returns it)."""
    import torch
    from fcb200 import _lib
    s = fcb.FCC(A_LAT, "Ar", CELLS)
    pot = fcb.LJ(SIGMA, EPS, R_CUT)
    calc = fcb.AnalyticalCalculator(TOL, R_CUT)
    n = 3 * s.n_atoms
    psi = julia_tensor((n, n, n), np.float64, device)
    psi32 = julia_tensor((n, n, n), np.float32, device)
    sp = int(stream.cuda_stream)

    def assemble():
        fcb.third_order_(psi, s, pot, calc, psi32_mw=psi32)

    asm = timed(assemble, stream, reps)
    dyn = fcb.dynamical_matrix(s, pot, calc, device=device)
    _, _, phi = fcb.get_modes(dyn, 3, phi32=True)
    k3_h = torch.empty(n ** 3, dtype=torch.float32).pin_memory()
    L = _lib.lib()
    h = _lib.handle(torch.device(device).index or 0)

    def blocked():
        _lib.check(L.fcb200_mcc3_blocked(h, int(psi32.data_ptr()), int(phi.data_ptr()), n, 256, _lib.FCB_MCC3_FP32,
                                         int(k3_h.data_ptr()), sp))

    blocked()
    t0 = time.perf_counter()
    for _ in range(reps):
        blocked()
    blk = (time.perf_counter() - t0) / reps
    del psi, psi32, k3_h
    torch.cuda.empty_cache()
    return {"workload": "perfect LJ FCC 4x4x4 (256 atoms), FP64 IFC3 + FP32 mass-weighted copy, FP32 mcc3 "
                        "block_size 256 (27 blocks) into pinned host memory",
            "assembly_s": asm, "mcc3_blocked_fp32_host_s": blk, "d2h_bytes": 4 * n ** 3,
            "checked": "tests/test_gpu_configs.py::test_config1_perfect_lattice_fp32_blocked"}


def run_reference(args, rank, world):
    """Reference arm: the reference path restated — CPU third_order (oracle,
    all host threads) + serial mass weighting + Float32 cast, then the blocked
    mcc3 (block_size 256, 27 blocks, D2H per block) with cuBLAS FP32 (TF32 off)
    standing in for CUDA.jl + cuTENSOR on the same GPU."""
    if rank != 0:
        return
    import torch
    from oracle import oracle as O
    import fcb200 as fcb
    torch.backends.cuda.matmul.allow_tf32 = False
    s = fcb.displaced(fcb.FCC(A_LAT, "Ar", CELLS), STD, SEED)
    n = 3 * s.n_atoms
    ifc2 = O.second_order_lj(s.positions, s.box_sizes, SIGMA, EPS, R_CUT, TOL)
    _, phi = O.get_modes(O.dynamical_matrix(ifc2, s.masses))
    phi_d = torch.from_numpy(np.ascontiguousarray(phi.astype(np.float32))).cuda()
    b = 256
    k3_host = torch.empty(n ** 3, dtype=torch.float32).numpy()

    def step():
        psi = O.third_order_lj(s.positions, s.box_sizes, SIGMA, EPS, R_CUT, TOL)
        O.mass_weight_third_order(psi, s.masses)
        psi32 = psi.astype(np.float32, order="F")
        del psi
        # [i,j,k] semantics: a Fortran array viewed through numpy keeps indices.
        dpsi = torch.from_numpy(np.ascontiguousarray(psi32.transpose(2, 1, 0))).cuda()  # [k,j,i] row-major
        del psi32
        out = k3_host.reshape((n, n, n), order="F")
        # mcc.jl:102-114: every block contracts all of Ψ with column-sliced φ
        # (mcc3_blocked!, mcc.jl:129-131), then copies the block to the host.
        for a0 in range(0, n, b):
            for b0 in range(0, n, b):
                for c0 in range(0, n, b):
                    k1 = torch.matmul(dpsi, phi_d[:, a0:a0 + b])                  # [k,j,p]
                    k2 = torch.einsum("kjp,jq->kpq", k1, phi_d[:, b0:b0 + b])     # [k,p,q]
                    del k1
                    k3 = torch.einsum("kpq,kr->pqr", k2, phi_d[:, c0:c0 + b])     # [p,q,r]
                    out[a0:a0 + b, b0:b0 + b, c0:c0 + b] = k3.cpu().numpy()
        torch.cuda.synchronize()

    steps, warm = min(args.steps, 3), min(args.warmup, 1)
    for _ in range(warm):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = (time.perf_counter() - t0) / steps
    line = {"metric": METRIC, "value": dt, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": dt * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": "LJ FCC 4x4x4 (256 atoms, n=768), displaced std 0.05 A seed 1234; "
                                   "CPU third_order+mass_weight+cast, then blocked FP32 mcc3 (block 256)",
                       "mcc3_standin": "torch/cuBLAS FP32, TF32 off, 27 blocks with D2H per block"},
            "cpu_baseline": {"value": dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                             "sample": "one full snapshot per step (oracle CPU assembly + cuBLAS FP32 blocked mcc3)"},
            "e2e": {"value": dt, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "tf32x3", "fp32"])
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline leg")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-batch", action="store_true", help="omit the 48-snapshot batch configuration")
    ap.add_argument("--skip-extra", action="store_true",
                    help="omit the other configurations (SW snapshot, adjoint, plain FP32 blocked) and the GEMM peaks")
    ap.add_argument("--out-dir", default=None,
                    help="directory for the clock samples and the autotune cache (default: a temporary directory)")
    ap.add_argument("--cells", default=None, help="FCC cells 'x,y,z' (profiling cases; default 4,4,4)")
    ap.add_argument("--minimal", action="store_true",
                    help="warm-up + timed steps only (for profiler captures of small cases)")
    args = ap.parse_args()
    if args.cells:
        global CELLS
        CELLS = tuple(int(c) for c in args.cells.split(","))

    from fcb200 import replicas
    rank, world, local = replicas.env_rank()
    import torch
    torch.cuda.set_device(local)
    if args.impl == "reference":
        # rank 0 alone runs the reference path; other ranks exit without work
        # and without joining any collective.
        if rank == 0:
            run_reference(args, rank, world)
        return
    pg = replicas.init("nccl", timeout_s=120)
    args.warmup = max(args.warmup, 3)
    out_dir = args.out_dir or tempfile.mkdtemp(prefix="fcb200_bench_")
    os.makedirs(out_dir, exist_ok=True)


    import fcb200 as fcb
    from fcb200 import _lib
    L = _lib.lib()
    dev = f"cuda:{local}"
    s, pot, calc, phi32 = build_workload(fcb, dev)
    n = 3 * s.n_atoms
    stream = torch.cuda.current_stream()
    sp = int(stream.cuda_stream)
    h = _lib.handle(local)
    d_pos = torch.from_numpy(s.positions).to(dev)
    d_box = torch.from_numpy(s.box_sizes).to(dev)
    d_m = torch.from_numpy(s.masses).to(dev)
    d_phi = torch.from_numpy(phi32).to(dev)
    psi64 = julia_tensor((n, n, n), np.float64, dev)
    k3 = julia_tensor((n, n, n), np.float32, dev)
    prec = _lib.PRECISIONS[args.precision]

    def step(precision=prec, k3_ptr=None, phi_ptr=None, pos_ptr=None, psi_ptr=None):
        _lib.check(L.fcb200_snapshot_lj(
            h, pos_ptr or int(d_pos.data_ptr()), s.n_atoms, int(d_box.data_ptr()), SIGMA, EPS, R_CUT, TOL,
            int(d_m.data_ptr()), phi_ptr or int(d_phi.data_ptr()), 0, n, precision, psi_ptr or int(psi64.data_ptr()),
            k3_ptr or int(k3.data_ptr()), sp))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    replicas.barrier(pg)
    clocks = Clocks(local, out_dir)
    clocks.start()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    clocks.wait_for(e1)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    replicas.barrier(pg)
    ms = replicas.max_over_ranks(ms, pg, device=dev)
    ms_per_step = ms / args.steps
    value = (ms / 1e3) / (args.steps * world)
    if args.minimal:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                              "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False,
                              "config": {"cells": list(CELLS), "n": n, "precision": args.precision},
                              "clocks": clk, "minimal": True}), flush=True)
        replicas.finalize(pg)
        return

    # ---- per-phase device times (profiled pass, same stream, outside the timed region)
    def profile_phases(precision, reps=3):
        _lib.check(L.fcb200_set_profiling(h, 1))
        acc = np.zeros(6)
        for _ in range(reps):
            step(precision=precision)
            out = (ctypes.c_double * 6)()
            _lib.check(L.fcb200_phase_times(h, out, 6))
            acc += np.array(out[:])
        _lib.check(L.fcb200_set_profiling(h, 0))
        return acc / reps

    phases = profile_phases(prec)
    gemm = None if args.skip_extra else gemm_peaks(dev)
    split = args.precision != "fp32"
    if split:
        # profiled pass: the FP64 writer runs alone inside the second phase; the
        # timed steps run it beside mode product 2 on a second stream
        names = ["pair_tables", "neighbours_phi_split_and_ifc3_dense_write", "sparse_coefs", "sparse_mode_product_1",
                 "mode_product_2", "mode_product_3"]
    else:
        names = ["pair_tables", "ifc3_dense_write", "phi_split", "mode_product_1", "mode_product_2", "mode_product_3"]
    phase_ms = {k: round(float(v), 4) for k, v in zip(names, phases)}

    peaks, peak_src = load_peaks()
    cs = None  # (Mp, Kc) when the compact sparse products run
    if not split:
        mp_ms = float(np.mean(phases[3:6]))
        flops_launch = 2.0 * n ** 4
        ach = flops_launch / (mp_ms * 1e-3) / 1e12
        pk = gemm["fp32_tflops"] if gemm else None
        roof = {"bound": "fp32-simt", "achieved": round(ach, 2), "peak": pk, "unit": "TFLOP/s",
                "frac": round(ach / pk, 4) if pk else None, "traffic": None,
                "kernel": "mode_product_f32_kernel (FFMA), 3 launches/step", "flops_per_launch": flops_launch,
                "avg_launch_ms": round(mp_ms, 4),
                "peak_source": "measured FP32 GEMM (torch/cuBLAS, TF32 off) in this run, gemm_peaks"}
    else:
        # Dominant kernel: the 2-CTA tensor-core mode product.  In the compact form
        # (taken at 256 atoms) it is the third product, reading U2 MN-major with
        # symmetric tiles; otherwise P2 and P3 both run it with symmetric tiles.
        # The executed tensor flops count the live 256-row tiles only, ×3 for the split.
        cs = compact_shapes(n, n, sparse_cap(s.positions, s.box_sizes, R_CUT))
        if cs:
            Mp, Kc = cs
            mp_ms = float(phases[5])
            flops_launch = full_sym_executed_flops(Mp, n, n)
            p2_flops = inner_sym_executed_flops(n, n, Mp, Kc)
        else:
            mp_ms = float(np.mean(phases[4:6]))
            flops_launch = float(np.mean([sym_executed_flops(n * n, n, n, n), sym_executed_flops(n * n, n, n, n)]))
        # The step is milliseconds long and the timed region well under a second, so the
        # burst GEMM figure is the denominator; the sustained (power-capped) one is kept beside it.
        if args.precision == "bf16x3":
            pk, pks = peaks["bf16_tflops"], peaks["bf16_tflops_sustained"]
        else:   # tf32x3: the TF32 GEMM measured in this run
            pk, pks = (gemm["tf32_tflops"] if gemm else None), None
        ach = flops_launch / (mp_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": round(ach, 2), "peak": pk, "unit": "TFLOP/s",
                "frac": round(ach / pk, 4) if pk else None,
                "frac_of_sustained": round(ach / pks, 4) if pks else None,
                "traffic": NCU_TRAFFIC.get("mode_product_tc2_p3" if cs else "mode_product_tc2_sym")
                if (args.precision == "bf16x3" and n == 768) else None,
                "traffic_unit": "bytes/launch (ncu, DRAM read+write)",
                "kernel": (f"mode_product_tc2_kernel ({args.precision}, 2-CTA tcgen05, MN-major A, row tiles "
                           "a/256 <= b/256, K3 stored by its full symmetry), the third product" if cs else
                           f"mode_product_tc2_kernel ({args.precision}, 2-CTA tcgen05, symmetric tiles), "
                           "2 launches/step (P2, P3)"),
                "flops_per_launch": flops_launch, "avg_launch_ms": round(mp_ms, 4),
                "useful_flops_per_step": 6.0 * n ** 4,
                "peak_source": (f"{peak_src} bf16_tflops (burst; executed tensor flops = 3x per product for the split)"
                                if args.precision == "bf16x3" else
                                "measured TF32 GEMM (torch/cuBLAS) in this run, gemm_peaks; executed tensor flops "
                                "= 3x per product for the split")}
        if cs:
            p2_ms = float(phases[4])
            a2 = p2_flops / (p2_ms * 1e-3) / 1e12
            esz2 = 2 if args.precision == "bf16x3" else 4
            p2_tiles = 3 * s.n_atoms * (Mp // 256) * ((Mp // 256) + 1) // 2   # upper (p, q) tiles per (atom, kc)
            p2_bytes = 2.0 * esz2 * (Mp * n * Kc + s.n_atoms * n * Kc + p2_tiles * 256 * 256)
            roof["second_product"] = {
                "kernel": "mode_product_tc2_kernel, grouped by atom (K = Kc), tiles p/256 <= q/256 of U2 only "
                          "(symmetric in (p, q))", "Mp": Mp, "Kc": Kc, "flops_per_launch": p2_flops,
                "ms": round(p2_ms, 4),
                "achieved": round(a2, 2), "frac": round(a2 / pk, 4) if pk else None,
                "traffic": NCU_TRAFFIC.get("mode_product_tc2_p2") if (args.precision == "bf16x3" and n == 768)
                else None,
                # its epilogue's stores bound it: the algorithmic bytes (U1c and φK read, upper U2 tiles
                # written) against the HBM copy bandwidth
                "algorithmic_bytes": p2_bytes,
                "frac_of_hbm": round(p2_bytes / (p2_ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4)}
    asm_bytes = 8.0 * n ** 3 + (0.0 if split else 4.0 * n ** 3)
    asm_ms = float(phases[1])
    roof_asm = {"bound": "hbm", "achieved": round(asm_bytes / (asm_ms * 1e-3) / 1e9, 1), "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": round(asm_bytes / (asm_ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4),
                "traffic": NCU_TRAFFIC.get("ifc3_dense_psi64") if (split and n == 768) else None,
                "kernel": "ifc3_dense_kernel2 (FP64 Psi only; the phase also holds the neighbour lists and the phi split)",
                "bytes_per_launch": asm_bytes, "avg_launch_ms": round(asm_ms, 4)}
    sparse_p1 = None
    if split:
        if cs:   # compact U1 and the per-atom φ rows, hi + lo planes
            u1_bytes = 2.0 * (2 if args.precision == "bf16x3" else 4) * (Mp * n * Kc + s.n_atoms * n * Kc)
        else:    # hi + lo BF16 planes of the dense-layout U1
            u1_bytes = 4.0 * n ** 3
        p1_ms = float(phases[3])
        sparse_p1 = {"kernel": "sparse_p1m_kernel (compact, CUDA cores, FP32, U1c mode-fastest)" if cs else
                     "sparse_p1_kernel (CUDA cores, FP32)", "ms": round(p1_ms, 4),
                     "bytes_written": u1_bytes, "achieved_gbs": round(u1_bytes / (p1_ms * 1e-3) / 1e9, 1),
                     "frac_of_hbm": round(u1_bytes / (p1_ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4)}

    # ---- accuracy of the timed path vs FP64 (outside timing)
    torch.cuda.synchronize()
    ref = fp64_reference_k3(psi64, s.masses, phi32)
    acc_err = {args.precision: err_vs(k3, ref)}
    # FP32 GPU form for the "split-BF16 vs FP32 GPU" comparison
    fp32_info = None
    packed_info = None
    if args.precision != "fp32":
        k3f = julia_tensor((n, n, n), np.float32, dev)
        step(precision=_lib.FCB_MCC3_FP32, k3_ptr=int(k3f.data_ptr()))
        torch.cuda.synchronize()
        acc_err["fp32"] = err_vs(k3f, ref)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        nf = 3
        for _ in range(nf):
            step(precision=_lib.FCB_MCC3_FP32, k3_ptr=int(k3f.data_ptr()))
        f1.record(stream)
        torch.cuda.synchronize()
        fp32_s = f0.elapsed_time(f1) / nf / 1e3
        fp32_info = {"s_per_snapshot": fp32_s, "speedup_split_vs_fp32": fp32_s / (ms_per_step / 1e3)}
        # the FP32 SIMT mode product against the measured FP32 GEMM
        fph = profile_phases(_lib.FCB_MCC3_FP32, reps=1)
        f_ms = float(np.mean(fph[3:6]))
        f_ach = 2.0 * n ** 4 / (f_ms * 1e-3) / 1e12
        fp32_info["mode_product"] = {
            "kernel": "mode_product_f32_kernel (FFMA), dense, 3 launches/step", "avg_launch_ms": round(f_ms, 4),
            "flops_per_launch": 2.0 * n ** 4, "achieved_tflops": round(f_ach, 2),
            "frac_of_measured_fp32_gemm": round(f_ach / gemm["fp32_tflops"], 4) if gemm else None}
        # the same precision with every mode product dense (no sparse P1, no symmetric tiles)
        dense_prec = prec | _lib.FCB_MCC3_FORCE_DENSE
        step(precision=dense_prec, k3_ptr=int(k3f.data_ptr()))
        torch.cuda.synchronize()
        acc_err[args.precision + "_dense_products"] = err_vs(k3f, ref)
        f0.record(stream)
        for _ in range(nf):
            step(precision=dense_prec, k3_ptr=int(k3f.data_ptr()))
        f1.record(stream)
        torch.cuda.synchronize()
        fp32_info["dense_products_s_per_snapshot"] = f0.elapsed_time(f1) / nf / 1e3
        if cs:   # the same step with the opt-in packed K3 (device-resident)
            kpk = julia_tensor((fcb.packed_k3_count(n),), np.float32, dev)
            kp = prec | _lib.FCB_K3_PACKED
            step(precision=kp, k3_ptr=int(kpk.data_ptr()))
            pph = profile_phases(kp, reps=1)
            pk_fl = full_sym_executed_flops(cs[0], n, n, packed=True)
            packed_info = {"s_per_snapshot": timed(lambda: step(precision=kp, k3_ptr=int(kpk.data_ptr())), stream, nf),
                           "k3_floats": fcb.packed_k3_count(n), "third_product_ms": round(float(pph[5]), 4),
                           "third_product_flops": pk_fl,
                           "third_product_achieved_tflops": round(pk_fl / (float(pph[5]) * 1e-3) / 1e12, 2),
                           "note": "FCB_K3_PACKED: the third product stores only K3[p,q,s], p <= q <= s, and skips "
                                   "the mode tiles that hold none"}
            del kpk
        fp32_info["speedup_split_vs_fp32_both_dense"] = fp32_s / fp32_info["dense_products_s_per_snapshot"]
        if args.precision == "bf16x3" and not args.skip_extra:
            # TF32x3 on the same step: time, error and its third product against the measured TF32 GEMM
            tf = _lib.PRECISIONS["tf32x3"]
            step(precision=tf, k3_ptr=int(k3f.data_ptr()))
            torch.cuda.synchronize()
            acc_err["tf32x3"] = err_vs(k3f, ref)
            tf_s = timed(lambda: step(precision=tf, k3_ptr=int(k3f.data_ptr())), stream, nf)
            tph = profile_phases(tf, reps=1)
            t_ach = flops_launch / (float(tph[5]) * 1e-3) / 1e12 if cs else None
            fp32_info["tf32x3"] = {
                "s_per_snapshot": tf_s, "third_product_ms": round(float(tph[5]), 4),
                "third_product_achieved_tflops": round(t_ach, 2) if t_ach else None,
                "third_product_frac_of_measured_tf32_gemm": round(t_ach / gemm["tf32_tflops"], 4)
                if (t_ach and gemm) else None}
        del k3f
    del ref
    torch.cuda.empty_cache()

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.skip_e2e:
        pos_h = np.ascontiguousarray(s.positions)
        phi_h = torch.from_numpy(phi32.reshape(-1, order="F").copy()).pin_memory()
        k3_h = torch.empty(n ** 3, dtype=torch.float32).pin_memory()
        ne = max(3, min(args.steps, 5))
        step(k3_ptr=int(k3_h.data_ptr()), phi_ptr=int(phi_h.data_ptr()), pos_ptr=pos_h.ctypes.data)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ne):
            step(k3_ptr=int(k3_h.data_ptr()), phi_ptr=int(phi_h.data_ptr()), pos_ptr=pos_h.ctypes.data)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / ne
        e2e = {"value": e2e_s / world if world > 1 else e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(pos_h.nbytes + phi_h.numel() * 4),
               "d2h_bytes_per_step": int(k3_h.numel() * 4),
               "note": "fcb200_snapshot_lj with host positions, pinned host phi and pinned host K3; "
                       "FP64 Psi stays in device memory"}
        # the same call also returning the FP64 Ψ to (pinned) host memory, as third_order does
        psi_h = torch.empty(n ** 3, dtype=torch.float64).pin_memory()
        step(k3_ptr=int(k3_h.data_ptr()), phi_ptr=int(phi_h.data_ptr()), pos_ptr=pos_h.ctypes.data,
             psi_ptr=int(psi_h.data_ptr()))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ne):
            step(k3_ptr=int(k3_h.data_ptr()), phi_ptr=int(phi_h.data_ptr()), pos_ptr=pos_h.ctypes.data,
                 psi_ptr=int(psi_h.data_ptr()))
        torch.cuda.synchronize()
        e2e["with_psi64_to_host"] = {"value": (time.perf_counter() - t0) / ne, "unit": UNIT,
                                     "d2h_bytes_per_step": int(k3_h.numel() * 4 + psi_h.numel() * 8)}
        del psi_h
        # opt-in packed K3 (FCB_K3_PACKED): only the entries p <= q <= s come back
        if split:
            kp = prec | _lib.FCB_K3_PACKED
            kp_h = torch.empty(fcb.packed_k3_count(n), dtype=torch.float32).pin_memory()
            step(precision=kp, k3_ptr=int(kp_h.data_ptr()), phi_ptr=int(phi_h.data_ptr()), pos_ptr=pos_h.ctypes.data)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(ne):
                step(precision=kp, k3_ptr=int(kp_h.data_ptr()), phi_ptr=int(phi_h.data_ptr()),
                     pos_ptr=pos_h.ctypes.data)
            torch.cuda.synchronize()
            e2e["packed_k3"] = {"value": (time.perf_counter() - t0) / ne, "unit": UNIT,
                                "h2d_bytes_per_step": int(pos_h.nbytes + phi_h.numel() * 4),
                                "d2h_bytes_per_step": int(kp_h.numel() * 4),
                                "note": "FCB_K3_PACKED: the M(M+1)(M+2)/6 entries p <= q <= s of the symmetric K3"}
            del kp_h

    batch = None
    if not args.skip_batch:
        _lib.check(L.fcb200_trim(h))
        torch.cuda.empty_cache()
        batch = batch_config(fcb, args.precision, dev, out_dir)

    extra = {}
    if not args.skip_extra:
        _lib.check(L.fcb200_trim(h))
        torch.cuda.empty_cache()
        extra["sw_snapshot"] = sw_snapshot_config(fcb, dev, stream)
        extra["adjoint"] = adjoint_config(fcb, dev, stream, s, pot, calc)
        extra["plain_fp32_blocked"] = config1(fcb, dev, stream)
        extra["measured_gemm_peaks"] = gemm

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline(phi32)

    # split: pair, self, neighbour lists, phi split, coefficients, sparse P1, P2 with the dense
    # writer beside it (second stream), P3
    kernels_per_step = 9 if split else 6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+" + args.precision, "data": "synthetic",
        "config": {"workload": "LJ FCC 4x4x4 (256 atoms, n=768), displaced std 0.05 A (seed 1234), "
                               "IFC3 FP64 + mass-weighted split operand, mcc3 all 768 modes",
                   "precision": args.precision, "parallelism": f"replicas x{world}",
                   "l2": "working set > L2 (Psi64 3.6 GB, intermediates 1.8 GB each); no flush",
                   "algorithm": ("P1 neighbourhood-compact (CUDA cores), P2 grouped by atom and P3 MN-major, "
                                 "both symmetric tensor-core tiles" if cs else
                                 "P1 block-sparse (CUDA cores), P2/P3 symmetric tensor-core tiles") if split
                   else "dense FP32 mode products"},
        "roofline": roof, "roofline_assembly": roof_asm, "sparse_p1": sparse_p1, "phase_ms": phase_ms,
        "overlap": ({"phase_sum_ms": round(float(phases.sum()), 4), "ms_per_step": round(ms_per_step, 4),
                     "saved_ms": round(float(phases.sum()) - ms_per_step, 4),
                     "note": "phase_ms from a profiled pass with every kernel alone; the timed steps run the "
                             "FP64 writer on a second stream beside the last tensor-core product(s)"}
                    if split else None),
        "error_vs_fp64": acc_err, "fp32_gpu": fp32_info, "packed_k3": packed_info, "clocks": clk, "e2e": e2e,
        "cpu_baseline": cpu, "batch": batch, "gpu_launches": kernels_per_step * args.steps,
    }
    line.update(extra)
    if rank == 0:
        print(json.dumps(line), flush=True)
    replicas.finalize(pg)


if __name__ == "__main__":
    main()
