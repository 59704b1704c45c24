"""Benchmark: fused-gate statevector simulation on B200 (one JSON line).

Workload (the 30-qubit configuration of the reference comparison): a random
brickwork circuit on 30 qubits, depth 20 (U3 on every qubit per layer, then
CZ on alternating neighbour pairs), started from |0...0>, fused with the
reference's size-only fusion at width k (default 4), complex128 statevector
(16 GiB, larger than L2).  One step = reset to |0...0> + every fused gate once.

  value  : algorithmic HBM bytes / s over the K timed steps, measured through
           the drop-in C ABI (compile_gate_ptx -> cubin_load -> kernel_launch)
           on a device-resident statevector.  Bytes per fused-gate pass are
           2 * 2^n * 16 (read + write, the reference's accounting,
           src/profile.rs:427-436).
  e2e    : same metric through the public Simulator API per step: gate
           matrices uploaded from host, run, <Z_q> for every qubit read back.
  roofline / cpu_baseline / clocks: see the JSON keys.

Keys beside the headline (rank 0, one GPU): c2_complex64 (the same 30-qubit
circuit in complex64, with its own roofline), qft (22-qubit QFT-CX), fusion_sweep
(k = 2..7, both precisions, tensor cores at k = 5, 6), tensor_path, largest_fit
(34-qubit complex64 / 33-qubit complex128, fidelity of a 28-qubit prefix against
the FP64 CPU restatement run in the same process), trajectories (persistent
kernel vs host-driven plain path vs exact density matrix) and serving (Poisson
streams at swept rates vs the same engine one request at a time).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
       [--precision f64|f32] [--k 4] [--n 30] [--depth 20]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def measured_peak_bf16():
    """Dense BF16 TFLOP/s (burst) from MEASURED_PEAKS.json, else an earlier
    cuBLAS measurement on a B200 (1590)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def build_fused(n: int, depth: int, k: int, seed: int = 2024):
    """The brickwork construction fused at width k by the native planner (the
    same decisions as fusion.optimize, tests/test_native_fusion.py)."""
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.types import QuantumCircuit

    circ = QuantumCircuit.brickwork(n, depth, seed)
    return circ, optimize_native(n, circ.gates(), FusionConfig.size_only(k)).gates()


_CB_LIB = None


def _cpu_baseline_lib():
    """The threaded SIMD CPU restatement of CAST's CPU kernels (oracle/), built
    on first use: the timed CPU baseline, and the FP64 result the GPU output is
    compared with.  It is compiled here with -march=native for the host cores
    that run it; if that build fails, the portable x86-64-v3 build is used.
    Returns (library, compiler flags)."""
    global _CB_LIB
    if _CB_LIB is not None:
        return _CB_LIB
    import ctypes as C

    from oracle import oracle as O

    O.build()
    flags, path = "-O3 -march=x86-64-v3", os.path.join(ROOT, "oracle", "build", "libcpu_baseline.so")
    try:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "native"], check=True,
                       capture_output=True, timeout=300)
        flags, path = "-O3 -march=native", os.path.join(ROOT, "oracle", "build",
                                                         "libcpu_baseline_native.so")
    except Exception:
        pass
    lib = C.CDLL(path)
    lib.cb_alloc.restype = C.c_void_p
    lib.cb_alloc.argtypes = [C.c_uint32, C.c_int]
    lib.cb_free.argtypes = [C.c_void_p]
    lib.cb_zero.argtypes = [C.c_void_p]
    lib.cb_store.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.cb_apply.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint32), C.c_uint32,
                             C.c_int]
    _CB_LIB = (lib, flags)
    return _CB_LIB


def cpu_reference_state(n: int, gates, threads: int) -> np.ndarray:
    """Final amplitudes (complex128) of a gate list applied to |0...0> by the FP64
    CPU restatement of CAST's statevector path, with `threads` host threads."""
    import ctypes as C

    lib, _ = _cpu_baseline_lib()
    sv = lib.cb_alloc(n, 0)
    if not sv:
        raise MemoryError("cpu reference allocation failed")
    try:
        lib.cb_zero(sv)
        for g in gates:
            m = np.ascontiguousarray(g.matrix()).view(np.float64)
            q = np.asarray(g.qubits(), dtype=np.uint32)
            lib.cb_apply(sv, m.ctypes.data_as(C.POINTER(C.c_double)),
                         q.ctypes.data_as(C.POINTER(C.c_uint32)), q.size, threads)
        ref = np.empty(1 << n, dtype=np.complex128)
        lib.cb_store(sv, ref.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    finally:
        lib.cb_free(sv)
    return ref


def fidelity_vs(ref: np.ndarray, psi: np.ndarray) -> dict:
    """1 - |<ref|psi>| (psi renormalised), max amplitude error and norm drift."""
    nrm = float(np.linalg.norm(psi))
    ov = abs(np.vdot(ref, psi)) / (float(np.linalg.norm(ref)) * nrm)
    return {"one_minus_abs_overlap": float(1.0 - ov), "max_abs_err": float(np.max(np.abs(ref - psi))),
            "norm_drift": float(1.0 - nrm)}


def cpu_parity(n: int, depth: int, k: int, precision: str, threads: int) -> dict:
    """Parity of the GPU result against CAST's FP64 CPU statevector path (its
    restatement in oracle/): the benchmark's brickwork construction at n qubits,
    fused at width k, run once from |0> on the CPU in FP64 and on the GPU in the
    benchmark's precision through the public gate-program API."""
    from cast_simulator_b200 import cuda as cu

    _, gates = build_fused(n, depth, k)
    ref = cpu_reference_state(n, gates, threads)
    prec = cu.CudaPrecision.F64 if precision == "f64" else cu.CudaPrecision.F32
    _, gsv = _run_fused(n, gates, prec, reps=1)
    psi = gsv.download()
    rep = fidelity_vs(ref, psi)
    return {"workload": f"brickwork-{n}q-d{depth} fused k={k} ({len(gates)} passes), from |0>",
            "reference": "FP64 CPU restatement of CAST's statevector path",
            "one_minus_abs_overlap": rep["one_minus_abs_overlap"], "max_abs_err": rep["max_abs_err"]}


def cpu_baseline_run(n: int, gates, precision: str, budget_s: float, threads: int):
    """Time the threaded SIMD CPU restatement (oracle/cpu_baseline.cpp) on the
    host cores: as many fused-gate passes as fit in the budget.  Returns
    (GB/s, passes, seconds)."""
    import ctypes as C

    lib, _ = _cpu_baseline_lib()
    f32 = precision == "f32"
    sv = lib.cb_alloc(n, int(f32))
    if not sv:
        raise MemoryError("cpu baseline allocation failed")
    lib.cb_zero(sv)
    amp_bytes = 8 if f32 else 16
    mats = [(np.ascontiguousarray(g.matrix()).view(np.float64), np.asarray(g.qubits(), dtype=np.uint32))
            for g in gates]
    # one untimed warm-up pass (page faults)
    m, q = mats[0]
    lib.cb_apply(sv, m.ctypes.data_as(C.POINTER(C.c_double)), q.ctypes.data_as(C.POINTER(C.c_uint32)),
                 q.size, threads)
    passes, t0 = 0, time.perf_counter()
    while True:
        m, q = mats[passes % len(mats)]
        lib.cb_apply(sv, m.ctypes.data_as(C.POINTER(C.c_double)),
                     q.ctypes.data_as(C.POINTER(C.c_uint32)), q.size, threads)
        passes += 1
        el = time.perf_counter() - t0
        if el >= budget_s and passes >= 2:
            break
    lib.cb_free(sv)
    return passes * 2 * (1 << n) * amp_bytes / el / 1e9, passes, el


def run_reference(args):
    """--impl reference: the reference's CPU path (threaded C++ restatement of
    CAST's CPU SIMD kernels; CAST itself cannot be built here) on the host cores,
    on the same 30-qubit configuration as the GPU arm."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n_cpu = min(args.n, args.cpu_n)
    _, gates = build_fused(n_cpu, args.depth, args.k)
    _, flags = _cpu_baseline_lib()
    samples = []
    for _ in range(args.warmup):
        cpu_baseline_run(n_cpu, gates, args.precision, args.cpu_budget / 4, threads)
    passes_tot, el_tot = 0, 0.0
    for _ in range(args.steps):
        gbs, passes, el = cpu_baseline_run(n_cpu, gates, args.precision, args.cpu_budget, threads)
        samples.append(gbs)
        passes_tot += passes
        el_tot += el
    v = float(np.mean(samples))
    sample = (f"{n_cpu}-qubit brickwork depth {args.depth} fused k={args.k}, "
              f"{passes_tot} fused-gate passes over {args.steps} steps of ~{args.cpu_budget:g} s")
    line = {
        "impl": "reference", "metric": "HBM GB/s (fused-gate statevector passes)", "value": v,
        "unit": "GB/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el_tot / max(args.steps, 1) * 1e3, "higher_is_better": True,
        "scaling": "weak", "dtype": args.precision, "data": "synthetic",
        "config": {"workload": f"brickwork-{args.n}q-d{args.depth}-{'c128' if args.precision == 'f64' else 'c64'}"
                   f"-k{args.k}", "cpu_sample_qubits": n_cpu},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": sample, "build": flags,
                         "stddev": float(np.std(samples, ddof=1)) if len(samples) > 1 else 0.0},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "vs_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


def _random_state(n: int, seed: int) -> np.ndarray:
    """Seeded i.i.d. Gaussian real/imaginary parts, normalised (complex128)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


def _run_fused(n: int, gates, precision, split: bool = False, initial=None, reps: int = 3,
               warm: bool = True, use_graph: bool = True):
    """Device time (median of reps, CUDA events) of a fused gate list as one
    gate program, and the final statevector object.  With `warm`, one untimed
    run first (graph capture, first launches); every timed run starts from the
    same initial state."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.simulator import Event, GateProgram, Stream

    prog = GateProgram(precision, n, 1e-12 if precision == cu.CudaPrecision.F64 else 1e-6,
                       1e-12 if precision == cu.CudaPrecision.F64 else 1e-6, split)
    for g in gates:
        prog.add(g.matrix(), g.qubits())
    sv = cu.CudaStatevector(n, precision)
    st = Stream()
    e0, e1 = Event(), Event()
    ts = []
    for rep in range(reps + (1 if warm else 0)):
        if initial is None:
            sv.zero(st)
        else:
            sv.upload(initial)
        e0.record(st)
        prog.run(sv, st, use_graph=use_graph)
        e1.record(st)
        e1.sync()
        if rep or not warm:
            ts.append(e1.elapsed_s(e0))
    return float(np.median(ts)), sv


def qft_leg(n: int = 22, seed: int = 7):
    """Plain method, small configuration: QFT-CX on a seeded random complex128
    state with the default fusion (size-only, k <= 6), against the same circuit
    unfused (fusion invariance; the oracle comparison is tests/test_gpu_configs.py)."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.types import QuantumCircuit

    circ = QuantumCircuit.qft_cx(n)
    init = _random_state(n, seed)
    fused = optimize_native(n, circ.gates(), FusionConfig.default()).gates()
    t, sv = _run_fused(n, fused, cu.CudaPrecision.F64, initial=init)
    got = sv.download()
    _, sv_u = _run_fused(n, circ.gates(), cu.CudaPrecision.F64, initial=init, reps=1)
    ref = sv_u.download()
    passes = len(fused)
    from collections import Counter

    from cast_simulator_b200.simulator import gate_engine

    engines = Counter(gate_engine(g.matrix(), g.qubits(), n, cu.CudaPrecision.F64) for g in fused)
    return {"workload": f"qft-cx-{n}q-c128-default-fusion", "unfused_gates": len(circ),
            "fused_gates": passes, "engines": dict(engines), "ms": t * 1e3,
            "hbm_gbs": passes * 2 * (1 << n) * 16 / t / 1e9,
            "gates_amps_per_s": len(circ) * (1 << n) / t,
            "max_abs_diff_vs_unfused": float(np.max(np.abs(got - ref)))}


def largest_leg(threads: int, depth: int = 10, n64: int = 34, n128: int = 33, n_prefix: int = 28):
    """Largest single-GPU fit: 34-qubit complex64 and 33-qubit complex128 (128 GiB
    each), random brickwork (depth 10) and QFT-CX; the plain CUDA-core path at
    k = 4 against split-precision programs (dense 5- and 6-qubit gates on the
    tensor cores) at k = 5, 6 for complex64.  Each run is one timed pass of the
    whole circuit after the state is reset (seconds-long, eager launches).
    Fidelity: the same constructions on a 28-qubit prefix, run once on the FP64
    CPU restatement of CAST's statevector path in this process and on the GPU in
    every variant."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.types import QuantumCircuit

    peak = measured_peak_hbm()[0]
    out = {"runs": [], "no_k7_tensor_form": "a 7-qubit gate's split operand (256 KB) is the MMA's "
           "shared-memory operand and does not fit there; k = 7 runs on the CUDA cores only"}
    for n, prec, label in ((n64, cu.CudaPrecision.F32, "c64"), (n128, cu.CudaPrecision.F64, "c128")):
        amp = 8 if label == "c64" else 16
        for name, circ in (("brickwork", QuantumCircuit.brickwork(n, depth, 2024)),
                           ("qft-cx", QuantumCircuit.qft_cx(n))):
            # complex64: the split-precision tensor path at k = 5, 6; complex128: the
            # QFT-CX fused at k = 6 runs its sparse blocks on the CSR kernels
            variants = [(4, False)] + ([(5, True), (6, True)] if label == "c64" else
                                       [(6, False)] if name == "qft-cx" else [])
            base = None
            for k, split in variants:
                fused = optimize_native(n, circ.gates(), FusionConfig.size_only(k)).gates()
                t, sv = _run_fused(n, fused, prec, split, reps=1, warm=False, use_graph=False)
                del sv
                gbs = len(fused) * 2 * (1 << n) * amp / t / 1e9
                base = base or t
                wl = f"{name}-{n}q" + (f"-d{depth}" if name == "brickwork" else "") + f"-{label}"
                out["runs"].append({"workload": wl, "fusion_k": k,
                                    "tensor_cores": split, "fused_gates": len(fused), "ms": t * 1e3,
                                    "hbm_gbs": gbs, "hbm_frac": gbs / peak,
                                    "speedup_vs_plain_k4": base / t})
    fid = {}
    t0 = time.perf_counter()
    for name, circ in (("brickwork", QuantumCircuit.brickwork(n_prefix, depth, 2024)),
                       ("qft-cx", QuantumCircuit.qft_cx(n_prefix))):
        g4 = optimize_native(n_prefix, circ.gates(), FusionConfig.size_only(4)).gates()
        ref = cpu_reference_state(n_prefix, g4, threads)
        for label, prec, k, split in (("c128-k4", cu.CudaPrecision.F64, 4, False),
                                      ("c64-k4", cu.CudaPrecision.F32, 4, False),
                                      ("c64-k5-tensor", cu.CudaPrecision.F32, 5, True),
                                      ("c64-k6-tensor", cu.CudaPrecision.F32, 6, True)):
            gk = g4 if k == 4 else optimize_native(n_prefix, circ.gates(), FusionConfig.size_only(k)).gates()
            _, sv = _run_fused(n_prefix, gk, prec, split, reps=1, warm=False, use_graph=False)
            psi = sv.download()
            del sv
            fid[f"{name}-{label}"] = fidelity_vs(ref, psi)
            del psi
        del ref
    out["fidelity_28q_prefix_vs_cpu_fp64"] = fid
    out["fidelity_reference"] = (f"FP64 CPU restatement of CAST's statevector path, {threads} host "
                                 f"threads, {time.perf_counter() - t0:.1f} s for both prefix circuits "
                                 "with the GPU runs")
    return out


def trajectory_leg(n: int = 16, depth: int = 30, n_traj: int = 4096, k: int = 3, n_plain: int = 48):
    """Noisy-trajectory configuration: brickwork depth 30 with depolarizing 1e-3
    after every gate and amplitude damping 5e-4 per qubit per layer, 4096
    trajectories in one persistent launch (CUDA graph).  Time to solution for
    <Z_q> on the same GPU against
      * the plain path one trajectory at a time (fused segments replayed as CUDA
        graphs, host draws, one masked FP64 reduction per damping layer), timed
        on n_plain trajectories;
      * the exact density matrix on the plain kernels (2n = 32 virtual qubits,
        complex64, 32 GiB), which has no statistical error.
    The trajectory mean is also checked against that exact <Z_q>."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.simulator import GateProgram, Stream
    from cast_simulator_b200.trajectory import TrajectoryProgram, run_plain_fused
    from cast_simulator_b200.types import QuantumCircuit

    circ = QuantumCircuit.brickwork(n, depth, 31337, depolarizing=1e-3, damping=5e-4)
    prog = TrajectoryProgram(circ, k)
    st = Stream()
    prog.run(n_traj, 1, st)
    times = []
    z = None
    for r in range(3):
        t0 = time.perf_counter()
        z, _ = prog.run(n_traj, 2 + r, st)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    mean = z.mean(axis=0)
    sig = z.std(axis=0, ddof=1)
    se = sig / np.sqrt(n_traj)
    rate = n_traj / t
    # every fused block is one pass over the trajectory's 2^n complex64 amplitudes
    # (read + write); the passes run out of L2, so this is an equivalent rate
    equiv = n_traj * prog.stats.n_blocks * 2 * (1 << n) * 8 / t / 1e9
    out = {"config": f"brickwork-{n}q-d{depth}, depolarizing 1e-3, damping 5e-4, c64, k={k}",
           "n_traj": n_traj, "seconds": t, "traj_per_s": rate, "pass_equivalent_gbs": equiv,
           "blocks": prog.stats.n_blocks, "error_sites": prog.stats.n_errors,
           "z_stderr_max": float(se.max()), "z_mean_first4": [float(x) for x in mean[:4]]}

    # plain path, one trajectory at a time
    run_plain_fused(circ, 2, 3, fusion_k=4, stream=st)  # warm: segment graphs, first launches
    t0 = time.perf_counter()
    zp = run_plain_fused(circ, n_plain, 5, fusion_k=4, stream=st)
    tp = (time.perf_counter() - t0) / n_plain
    out["plain_per_trajectory"] = {
        "method": "plain gate kernels, one trajectory at a time: fused unitary segments (k=4) "
                  "replayed as CUDA graphs, host Pauli draws, one FP64 masked reduction per "
                  "damping layer",
        "n_traj": n_plain, "traj_per_s": 1.0 / tp, "seconds_for_4096": 4096 * tp,
        "persistent_speedup": rate * tp,
        "z_mean_first4": [float(x) for x in zp.mean(axis=0)[:4]]}

    # exact density matrix on the plain kernels
    sup = [g.to_density_matrix_gate(n) for g in circ.gates()]
    fused = optimize_native(2 * n, sup, FusionConfig.size_only(4))
    gp = GateProgram(cu.CudaPrecision.F32, 2 * n, 1e-6, 1e-6)
    from cast_simulator_b200 import _lib as L

    eb = L.errbuf()
    L.check(L.lib().cast_b200_program_add_fused(gp.handle, fused.handle, eb, L.ERR_LEN), eb,
            "program_add_fused")
    rho = cu.CudaStatevector(2 * n, cu.CudaPrecision.F32)
    from cast_simulator_b200.simulator import Event

    e0, e1 = Event(), Event()
    rho.zero(st)
    e0.record(st)
    gp.run(rho, st, use_graph=False)
    e1.record(st)
    e1.sync()
    t_dm = e1.elapsed_s(e0)
    pops = np.zeros(1 << n)
    L.check(L.lib().cast_b200_dm_populations(rho.dptr, n, 0, pops.ctypes.data_as(L.c_dp), st.handle,
                                             eb, L.ERR_LEN), eb, "dm_populations")
    del rho
    idx = np.arange(1 << n)
    z_dm = np.array([1 - 2 * pops[(idx >> q) & 1 == 1].sum() for q in range(n)]) / pops.sum()
    dev = np.abs(mean - z_dm)
    dm_passes = len(fused)
    out["density_matrix_exact"] = {
        "method": f"2n = {2 * n} virtual qubits, complex64 ({(8 << (2 * n)) / 2**30:.0f} GiB), "
                  "superoperators fused at k=4 on the plain kernels",
        "fused_passes": dm_passes, "seconds": t_dm,
        "hbm_gbs": dm_passes * 2 * (8 << (2 * n)) / t_dm / 1e9,
        "trajectory_mean_max_dev": float(dev.max()),
        "trajectory_mean_max_dev_in_stderr": float((dev / se).max())}
    # time to solution at a target standard error eps of every <Z_q>:
    # trajectories need max_q sigma_q^2 / eps^2 runs; the density matrix is exact
    eps = float(se.max())
    out["time_to_solution"] = {
        "target_stderr": eps,
        "persistent_kernel_s": t, "plain_per_trajectory_s": 4096 * tp, "density_matrix_s": t_dm,
        "stderr_where_persistent_equals_dm": float(sig.max() / np.sqrt(rate * t_dm))}
    return out


def sampling_leg(n: int = 30, depth: int = 20, n_shots: int = 1_000_000, k: int = 4):
    """On-device shot sampling of the 30-qubit brickwork state (complex128, 16 GiB):
    n_shots full bitstrings by the inverse CDF (cast_b200_sample), against the
    reference's method on the same state - download the statevector, build the
    FP64 CDF on the host, binary-search it per shot (src/simulator/mod.rs:282-291,
    measure.rs:49-76), timed here with numpy.  The device reads the state once
    for the chunk totals and once more for the chunks that receive shots."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.simulator import Event, Stream, sample

    import torch

    _, gates = build_fused(n, depth, k)
    _, sv = _run_fused(n, gates, cu.CudaPrecision.F64, reps=1, warm=False, use_graph=False)
    st = Stream()
    sample(sv, 1000, seed=1, stream=st)  # first launches
    # the keys land in one reused page-locked buffer: a direct DMA, no driver staging
    keys = torch.empty(n_shots, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    e0, e1 = Event(), Event()
    ts = []
    for r in range(5):
        e0.record(st)
        sample(sv, n_shots, seed=10 + r, stream=st, out=keys)
        e1.record(st)
        e1.sync()
        ts.append(e1.elapsed_s(e0))
    t = float(np.median(ts))
    state_bytes = (1 << n) * 16
    out = {"workload": f"brickwork-{n}q-d{depth}-c128 final state, {n_shots} shots",
           "ms": t * 1e3, "ms_runs": [x * 1e3 for x in ts], "shots_per_s": n_shots / t,
           "state_reads_gbs": 2 * state_bytes / t / 1e9,
           "output": "keys copied to a reused page-locked host buffer",
           "distinct_outcomes": int(np.unique(keys).size)}
    t0 = time.perf_counter()
    psi = sv.download()
    t_dl = time.perf_counter() - t0
    del sv
    u = np.random.default_rng(3).random(n_shots)
    t1 = time.perf_counter()
    cdf = np.cumsum(psi.real * psi.real + psi.imag * psi.imag)
    del psi
    idx = np.minimum(np.searchsorted(cdf, u, side="right"), cdf.size - 1)
    t_host = time.perf_counter() - t1
    del cdf, idx
    out["host_inverse_cdf"] = {"method": "download + numpy FP64 cumsum + searchsorted (one thread)",
                               "download_s": t_dl, "cdf_and_search_s": t_host,
                               "total_s": t_dl + t_host, "device_speedup": (t_dl + t_host) / t}
    return out


def serving_leg(n_req: int, rates=(20.0, 80.0, 320.0)):
    """Serving stream (bounded sample of the 10,000-request configuration, same
    distributions): Poisson arrivals of random brickwork circuits, 10..28 qubits,
    depth 5..40, half complex64 / half complex128, 20% noisy (depolarizing 1e-3,
    256 trajectories; noisy circuits have at most 20 qubits, the trajectory
    kernel's range).  At each swept rate: p50/p99 latency and circuits/s of
      * the engine: continuous batching, small pure requests (<= 16 qubits) on
        the batcher thread (together in the circuit-batch kernel when 32 or more
        wait, else one after another on the plain kernels), the rest on worker
        streams, complex64 requests of 20+ qubits as split-precision programs on
        the tensor cores;
      * the same engine with the circuit-batch kernel off;
      * sequential execution on the plain path: the same engine one request at a
        time (max_slots = 1, no batching, no tensor cores), on the same arrivals.
    Latency percentiles are also given per request class (pure <= 16 qubits,
    pure 17..28, noisy).
    An unmeasured pass of the fastest stream warms each engine first (kernel
    module loads, first allocation of each pooled statevector size)."""
    from cast_simulator_b200 import serving as S

    def stream(rate):
        return S.make_stream(n_req, rate, 7, n_range=(10, 28), noisy_max_qubits=20)

    out = {"requests_per_rate": n_req, "n_range": [10, 28], "noisy_max_qubits": 20,
           "sample": f"{n_req} requests per rate of the 10,000-request stream's distributions",
           "rates": [{"rate_hz": r} for r in rates]}
    for label, kw in (("engine", {"max_slots": 8}),
                      ("engine_no_batch_kernel", {"max_slots": 8, "batch_max_qubits": 0}),
                      ("sequential", {"max_slots": 1, "batch_max_qubits": 0, "split_min_qubits": 0})):
        eng = S.ServingEngine(**kw)
        try:
            eng.run_stream(stream(max(rates)))
            for i, rate in enumerate(rates):
                eng.max_concurrent = 0
                b0, r0, p0 = eng.batches_run, eng.batched_requests, eng.small_plain_requests
                t0 = time.perf_counter()
                res = eng.run_stream(stream(rate))
                wall = time.perf_counter() - t0
                entry = {**S.latency_summary([r.latency for r in res]),
                         "circuits_per_s": n_req / wall, "max_concurrent": eng.max_concurrent,
                         "wall_s": wall}
                classes = {"pure_small": [r.latency for r in res if not r.n_traj and r.n_qubits <= 16],
                           "pure_large": [r.latency for r in res if not r.n_traj and r.n_qubits > 16],
                           "noisy": [r.latency for r in res if r.n_traj]}
                entry["by_class"] = {c: {"p50_ms": float(np.percentile(v, 50) * 1e3),
                                         "p99_ms": float(np.percentile(v, 99) * 1e3), "n": len(v)}
                                     for c, v in classes.items() if v}
                if eng.batches_run > b0 or eng.small_plain_requests > p0:
                    entry["batch_launches"] = eng.batches_run - b0
                    entry["batched_requests"] = eng.batched_requests - r0
                    entry["small_requests_on_plain_path"] = eng.small_plain_requests - p0
                if label == "engine":
                    out["rates"][i].update(entry)
                else:
                    out["rates"][i][label] = entry
        finally:
            eng.shutdown()
    for r in out["rates"]:
        r["p99_speedup_vs_sequential"] = r["sequential"]["p99_ms"] / r["p99_ms"]
        r["p99_speedup_vs_no_batch_kernel"] = r["engine_no_batch_kernel"]["p99_ms"] / r["p99_ms"]
    return out


def circuit_batch_leg(n_circ: int = 2048, n_range=(10, 16), depth_range=(5, 40), seed: int = 5):
    """Many small circuits (random brickwork, 10..16 qubits, depth 5..40, half
    complex64 / half complex128) in ONE persistent launch of the circuit-batch
    kernel (fusion k = 3, one CTA a circuit) against the plain path run circuit
    after circuit (each fused at k = 4 into a gate program replayed as a CUDA
    graph, <Z_q> by the FP64 device reduction): time to <Z_q> of every circuit,
    host fusion excluded on both sides."""
    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.simulator import CircuitBatch, GateProgram, Stream, qubit_populations
    from cast_simulator_b200.types import QuantumCircuit

    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_circ):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        d = int(rng.integers(depth_range[0], depth_range[1] + 1))
        prec = cu.CudaPrecision.F64 if i % 2 else cu.CudaPrecision.F32
        specs.append((n, prec, QuantumCircuit.brickwork(n, d, 9000 + i)))
    st = Stream()
    fused3 = [optimize_native(n, c.gates(), FusionConfig.size_only(3)) for n, _, c in specs]
    svs = [cu.CudaStatevector(n, p) for n, p, _ in specs]
    batch = CircuitBatch()
    for sv, f in zip(svs, fused3):
        batch.add(sv, f)
    batch.run(st)  # warm: buffers, first launch
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        zb = batch.run(st)
        ts.append(time.perf_counter() - t0)
    t_batch = float(np.median(ts))
    amps = sum(1 << n for n, _, _ in specs)
    # plain path, one circuit after another on the whole GPU
    progs = []
    for (n, prec, c), sv in zip(specs, svs):
        f4 = optimize_native(n, c.gates(), FusionConfig.size_only(4))
        tol = 1e-12 if prec == cu.CudaPrecision.F64 else 1e-6
        gp = GateProgram(prec, n, tol, tol)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_program_add_fused(gp.handle, f4.handle, eb, L.ERR_LEN), eb,
                "program_add_fused")
        progs.append(gp)

    def plain_all():
        zs = []
        for gp, sv in zip(progs, svs):
            sv.zero(st)
            gp.run(sv, st, use_graph=True)
            p1, nrm = qubit_populations(sv, st)
            zs.append((nrm - 2 * p1) / nrm)
        return zs

    plain_all()  # graph capture
    t0 = time.perf_counter()
    zp = plain_all()
    t_plain = time.perf_counter() - t0
    dev = max(float(np.max(np.abs(a - b))) for a, b in zip(zb, zp))
    return {"workload": f"{n_circ} random brickwork circuits, {n_range[0]}..{n_range[1]} qubits, "
                        f"depth {depth_range[0]}..{depth_range[1]}, half complex64 / half complex128",
            "batch_kernel_s": t_batch, "circuits_per_s": n_circ / t_batch,
            "amplitudes_per_s": amps / t_batch,
            "plain_sequential_s": t_plain, "plain_circuits_per_s": n_circ / t_plain,
            "speedup": t_plain / t_batch, "max_abs_z_diff_batch_vs_plain": dev}


def fusion_sweep_leg(n: int, depth: int):
    """The brickwork with fusion width k = 2..7 on the CUDA-core path in complex128
    and complex64, and on the split-BF16 tensor cores for k = 5, 6 (complex64):
    device time per circuit (median of 2 after a warm-up run), fused passes, and
    the HBM rate those passes imply."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.types import QuantumCircuit

    peak = measured_peak_hbm()[0]
    circ = QuantumCircuit.brickwork(n, depth, 2024)
    out = {"workload": f"brickwork-{n}q-d{depth}", "runs": []}
    cases = [(cu.CudaPrecision.F64, "c128", False, k) for k in range(2, 8)]
    cases += [(cu.CudaPrecision.F32, "c64", False, k) for k in range(2, 8)]
    cases += [(cu.CudaPrecision.F32, "c64", True, k) for k in (5, 6)]
    fused = {k: optimize_native(n, circ.gates(), FusionConfig.size_only(k)).gates() for k in range(2, 8)}
    for prec, label, split, k in cases:
        gates = fused[k]
        t, sv = _run_fused(n, gates, prec, split, reps=2)
        b_amp = 16 if label == "c128" else 8
        gbs = len(gates) * 2 * (1 << n) * b_amp / t / 1e9
        out["runs"].append({"precision": label, "tensor_cores": split, "fusion_k": k,
                            "fused_gates": len(gates), "ms_per_circuit": t * 1e3,
                            "hbm_gbs": gbs, "hbm_frac": gbs / peak})
        del sv
    for label in ("c128", "c64"):
        best = min((r for r in out["runs"] if r["precision"] == label),
                   key=lambda r: r["ms_per_circuit"])
        out[f"best_{label}"] = {"fusion_k": best["fusion_k"], "tensor_cores": best["tensor_cores"],
                                "ms_per_circuit": best["ms_per_circuit"]}
    return out


def tensor_leg(n: int, depth: int, sweep: dict):
    """Tensor-core fused path (complex64, split BF16, k = 5 and 6) against the
    plain CUDA-core path at its best width (k = 4) on the full 30-qubit brickwork,
    from the fusion sweep's runs; and 1 - |<psi_ref|psi>| against the FP64 CPU
    restatement of CAST's statevector path on a 24-qubit brickwork of the same
    construction."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.types import QuantumCircuit

    peak = measured_peak_hbm()[0]
    out = {"workload": f"brickwork-{n}q-d{depth}-c64", "runs": []}
    circ = QuantumCircuit.brickwork(n, depth, 2024)
    by_k = {}
    for r in sweep["runs"]:
        if r["precision"] == "c64" and (r["fusion_k"], r["tensor_cores"]) in ((4, False), (5, True), (6, True)):
            by_k[r["fusion_k"]] = r
    for k in (4, 5, 6):
        r = by_k[k]
        t = r["ms_per_circuit"] / 1e3
        run = {"fusion_k": k, "tensor_cores": r["tensor_cores"], "fused_gates": r["fused_gates"],
               "ms_per_circuit": r["ms_per_circuit"], "hbm_gbs": r["hbm_gbs"],
               "hbm_frac": r["hbm_gbs"] / peak}
        if r["tensor_cores"]:
            gates = optimize_native(n, circ.gates(), FusionConfig.size_only(k)).gates()
            # tensor-pipe work of the passes that ran there: 3 split products of the
            # real (2D x 2D) GEMM per group, D = 2^kg
            flops = sum(3 * 2 * (2 << g.n_qubits()) ** 2 * (1 << (n - g.n_qubits()))
                        for g in gates if g.n_qubits() in (5, 6))
            bf16 = measured_peak_bf16()
            run["tensor_tflops"] = flops / t / 1e12
            run["tensor_frac"] = flops / t / 1e12 / bf16 if bf16 else None
        out["runs"].append(run)
    base = out["runs"][0]["ms_per_circuit"]
    for r in out["runs"]:
        r["speedup_vs_plain_k4"] = base / r["ms_per_circuit"]
    nf = 24
    small = QuantumCircuit.brickwork(nf, depth, 2024)
    ref = cpu_reference_state(nf, optimize_native(nf, small.gates(), FusionConfig.size_only(4)).gates(),
                              os.cpu_count() or 1)
    fid = {}
    for k in (5, 6):
        g = optimize_native(nf, small.gates(), FusionConfig.size_only(k)).gates()
        _, sv = _run_fused(nf, g, cu.CudaPrecision.F32, True, reps=1, warm=False)
        fid[f"k{k}"] = fidelity_vs(ref, sv.download())
        del sv
    out["fidelity_24q_vs_cpu_fp64"] = fid
    return out


def traffic_from_profile(n: int, precision: str, k: int):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (captured on a smaller statevector and scaled by amplitudes)."""
    p = os.path.join(ROOT, "profiles", "gate_kernel_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d[f"{precision}_k{k}"]
        return e["dram_bytes_per_launch"] * (1 << n) / (1 << e["n_qubits"])
    except Exception:
        return None


def plain_line(n: int, depth: int, k: int, precision: str, steps: int, warmup: int, local: int,
               pg=None) -> dict:
    """The fused brickwork through the drop-in C ABI (compile_gate_ptx ->
    cubin_load -> kernel_launch per fused gate, the reference's execution path)
    on a device-resident statevector: `warmup` untimed steps, then `steps` timed
    steps bracketed by a barrier and CUDA events on the launching stream, with
    the SM clocks sampled meanwhile.  One step = reset to |0...0> + every fused
    gate once.  Returns the device time (max over ranks), per-kernel event times
    by gate size, and the fused circuit."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.simulator import Event

    prec = cu.CudaPrecision.F64 if precision == "f64" else cu.CudaPrecision.F32
    spec = cu.CudaKernelGenSpec.f64() if prec == cu.CudaPrecision.F64 else cu.CudaKernelGenSpec.f32()
    circ, gates = build_fused(n, depth, k)
    mgr = cu.CudaKernelManager(spec, timing=True)
    kids = [mgr.generate(g) for g in gates]
    sv = cu.CudaStatevector(n, prec)

    def step():
        sv.zero()
        for kid in kids:
            mgr.apply(kid, sv)
        return mgr.sync()

    for _ in range(warmup):
        step()
    stream = mgr.stream  # the launching stream: events bracket the kernels themselves
    if pg:
        pg.barrier()
    e_start, e_end = Event(), Event()
    per_kernel = {}
    with ClockSampler(local) as clk:
        e_start.record(stream)
        wall0 = time.perf_counter()
        for _ in range(steps):
            st = step()
            for kt in st.kernels:
                per_kernel.setdefault(kt.n_gate_qubits, []).append(kt.gpu_time)
        e_end.record(stream)
        e_end.sync()
        wall = time.perf_counter() - wall0
    t = max(e_end.elapsed_s(e_start), 1e-12)
    if pg:
        import torch

        tt = torch.tensor([t], device=f"cuda:{local}", dtype=torch.float64)
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        t = float(tt.item())
    del sv
    return {"t": t, "per_kernel": per_kernel, "circ": circ, "gates": gates, "clocks": clk.summary(),
            "wall": wall, "n_launch": steps * len(gates)}


def roofline_of(run: dict, n: int, precision: str) -> dict:
    """The dominant kernel (the gate size with the largest summed device time):
    algorithmic bytes per launch / its average CUDA-event duration, against the
    measured HBM copy peak."""
    amp_bytes = 16 if precision == "f64" else 8
    per_kernel = run["per_kernel"]
    dom_k = max(per_kernel, key=lambda kk: sum(per_kernel[kk]))
    dom_avg = float(np.mean(per_kernel[dom_k]))
    achieved = 2 * (1 << n) * amp_bytes / dom_avg / 1e9
    peak, peak_kind = measured_peak_hbm()
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_from_profile(n, precision, dom_k), "kernel": f"k_gate k={dom_k}",
            "kernel_time_share": sum(per_kernel[dom_k]) / sum(sum(v) for v in per_kernel.values()),
            "peak_kind": peak_kind}


def sharded_line(args, ws: int, rank: int, local: int, pg) -> dict:
    """The brickwork on one statevector sharded over the N ranks (weak scaling:
    every rank holds 2^n amplitudes, the circuit has n + log2 N qubits), fused
    at width k; gates on global qubits are preceded by pairwise qubit-swap
    exchanges over NCCL, streamed through fixed staging buffers, with the
    look-ahead planner choosing what to evict.  Timed like the headline: warm-up
    runs, then `steps` runs bracketed by a barrier and CUDA events on the
    launching stream, max over ranks.  e2e: the same run with <Z_q> read back to
    the host every step (the gate matrices go from host to device every step)."""
    import torch

    from cast_simulator_b200 import distributed as D
    from cast_simulator_b200.simulator import Event

    g = ws.bit_length() - 1
    if 1 << g != ws:
        raise ValueError("the sharded statevector needs a power-of-two number of GPUs")
    n_tot = args.n + g
    circ, gates = build_fused(n_tot, args.depth, args.k)
    f64 = args.precision == "f64"
    dtype = torch.complex128 if f64 else torch.complex64
    shard = torch.zeros(1 << args.n, dtype=dtype, device=f"cuda:{local}")
    sv = D.ShardedStatevector(n_tot, shard, D.cuda_apply_local(1 if f64 else 0), group=None)

    def step():
        sv.set_zero()
        sv.apply_circuit(gates)

    # every launch of the run (torch ops, gate kernels, NCCL ordering) goes to one
    # non-default stream, the one the events are recorded on: the legacy default
    # stream has no handle an event can be recorded on through the C ABI
    st = torch.cuda.Stream(device=f"cuda:{local}")
    with torch.cuda.stream(st):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        ex0, amps0 = sv.n_exchanges, sv.exchanged_amps
        e0, e1 = Event(), Event()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            e0.record(st.cuda_stream)
            for _ in range(args.steps):
                step()
            e1.record(st.cuda_stream)
            e1.sync()
        t = max(e1.elapsed_s(e0), 1e-12)
        ex_step = (sv.n_exchanges - ex0) / max(1, args.steps)
        amps_step = (sv.exchanged_amps - amps0) / max(1, args.steps)
        if pg:
            tt = torch.tensor([t], device=f"cuda:{local}", dtype=torch.float64)
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
            t = float(tt.item())
        amp = 16 if f64 else 8
        bytes_per_pass = 2 * (1 << n_tot) * amp
        value = args.steps * len(gates) * bytes_per_pass / t / 1e9
        # e2e: <Z> back to the host every step
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
            z = sv.expectation_z()
        e2e_t = time.perf_counter() - t0
        torch.cuda.synchronize()
    if pg:
        et = torch.tensor([e2e_t], device=f"cuda:{local}", dtype=torch.float64)
        pg.all_reduce(et, op=pg.ReduceOp.MAX)
        e2e_t = float(et.item())
    return {
        "metric": "HBM GB/s (fused-gate statevector passes)", "value": value, "unit": "GB/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": {"workload": f"brickwork-{n_tot}q-d{args.depth}-{'c128' if f64 else 'c64'}-k{args.k}",
                   "n_qubits": n_tot, "shard_qubits": args.n, "depth": args.depth,
                   "fusion_k": args.k, "unfused_gates": len(circ), "fused_gates": len(gates),
                   "l2": "no flush: each shard is larger than L2",
                   "parallelism": f"sv-shard{ws}"},
        "exchange": {"per_step": ex_step, "amplitudes_per_step_per_rank": amps_step,
                     "bytes_per_step_per_rank": 2 * amps_step * amp},
        "e2e": {"value": args.steps * len(gates) * bytes_per_pass / e2e_t / 1e9, "unit": "GB/s",
                "h2d_bytes_per_step": sum(16 * gg.matrix().size for gg in gates),
                "d2h_bytes_per_step": 8 * (n_tot + 1)},
        "gpu_launches": args.steps * len(gates),
        "clocks": clk.summary(),
        "z_expectation_sample": [float(x) for x in z[:4]],
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--k", type=int, default=4)
    ap.add_argument("--n", type=int, default=30)
    ap.add_argument("--depth", type=int, default=20)
    ap.add_argument("--cpu-n", type=int, default=30)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip every leg beside the headline (and the CPU baseline)")
    ap.add_argument("--no-sweep", action="store_true", help="skip the fusion-width sweep k = 2..7")
    ap.add_argument("--no-largest", action="store_true",
                    help="skip the 34q complex64 / 33q complex128 largest-fit leg")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--sharded", action="store_true",
                    help="one statevector sharded over the GPUs (the default when N > 1)")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1: N independent replicas of the 30-qubit headline instead")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)

    ws, rank, local = dist_env()
    pg = None
    if ws > 1:
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        pg = dist

    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.simulator import Simulator

    eb = L.errbuf()
    L.check(L.lib().cast_b200_set_device(local, eb, L.ERR_LEN), eb, "set_device")
    if args.sharded or (ws > 1 and not args.replicas):
        line = sharded_line(args, ws, rank, local, pg)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return 0
    prec = cu.CudaPrecision.F64 if args.precision == "f64" else cu.CudaPrecision.F32
    spec = cu.CudaKernelGenSpec.f64() if prec == cu.CudaPrecision.F64 else cu.CudaKernelGenSpec.f32()
    amp_bytes = 16 if prec == cu.CudaPrecision.F64 else 8
    n = args.n
    bytes_per_pass = 2 * (1 << n) * amp_bytes

    # ---- value: drop-in C ABI path, device-resident statevector ----
    run = plain_line(n, args.depth, args.k, args.precision, args.steps, args.warmup, local, pg)
    t, gates, circ = run["t"], run["gates"], run["circ"]
    value = ws * args.steps * len(gates) * bytes_per_pass / t / 1e9

    # ---- e2e: public Simulator API, gates from host, <Z> read back ----
    from cast_simulator_b200.fusion import CircuitGraph

    sim = Simulator(spec)
    fused_graph = CircuitGraph.from_gates(n, gates)
    h2d = sum(16 * g.matrix().size for g in gates)
    d2h = 8 * (n + 1)
    sim.simulate(fused_graph).expectation_z()
    e0 = time.perf_counter()
    zs = None
    for _ in range(args.steps):
        state = sim.simulate(fused_graph)
        zs = state.expectation_z()
        del state
    e2e_t = time.perf_counter() - e0
    sim.release_memory()
    if pg:
        import torch

        et = torch.tensor([e2e_t], device=f"cuda:{local}", dtype=torch.float64)
        pg.all_reduce(et, op=pg.ReduceOp.MAX)
        e2e_t = float(et.item())
    e2e_value = ws * args.steps * len(gates) * bytes_per_pass / e2e_t / 1e9

    line = {
        "metric": "HBM GB/s (fused-gate statevector passes)",
        "value": value,
        "unit": "GB/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": args.precision,
        "data": "synthetic",
        "config": {
            "workload": f"brickwork-{n}q-d{args.depth}-{'c128' if args.precision == 'f64' else 'c64'}-k{args.k}",
            "n_qubits": n, "depth": args.depth, "fusion_k": args.k,
            "unfused_gates": len(circ), "fused_gates": len(gates),
            "statevector_bytes": (1 << n) * amp_bytes,
            "l2": "no flush: the statevector is larger than L2",
            "parallelism": f"replicas{ws}",
        },
        "gates_amps_per_s": ws * args.steps * len(gates) * (1 << n) / t,
        "roofline": roofline_of(run, n, args.precision),
        "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": run["n_launch"],
        "clocks": run["clocks"],
        "wall_s_timed": run["wall"],
        "z_expectation_sample": [float(x) for x in zs[:4]] if zs is not None else None,
    }
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        n_cpu = min(n, args.cpu_n)
        _, cgates = build_fused(n_cpu, args.depth, args.k)
        gbs, passes, el = cpu_baseline_run(n_cpu, cgates, args.precision, args.cpu_budget, threads)
        line["cpu_baseline"] = {
            "value": gbs, "unit": "GB/s", "cores": threads, "kind": "port",
            "build": _cpu_baseline_lib()[1],
            "sample": f"{passes} fused-gate passes of the {n_cpu}-qubit brickwork (k={args.k}) in {el:.1f} s",
            "parity": cpu_parity(min(n, 22), args.depth, args.k, args.precision, threads)}
    # the extra legs run on one GPU only: under torchrun the other ranks would sit
    # in the closing barrier for the minutes they take
    if rank == 0 and ws == 1 and not args.no_extras:
        threads = os.cpu_count() or 1
        other = "f32" if args.precision == "f64" else "f64"
        orun = plain_line(n, args.depth, args.k, other, min(args.steps, 10), 3, local)
        ob = 2 * (1 << n) * (16 if other == "f64" else 8)
        line["c2_" + ("complex64" if other == "f32" else "complex128")] = {
            "workload": f"brickwork-{n}q-d{args.depth}-{'c64' if other == 'f32' else 'c128'}-k{args.k}",
            "value": min(args.steps, 10) * len(orun["gates"]) * ob / orun["t"] / 1e9, "unit": "GB/s",
            "ms_per_step": orun["t"] / min(args.steps, 10) * 1e3, "dtype": other,
            "roofline": roofline_of(orun, n, other), "clocks": orun["clocks"]}
        import gc

        def leg(key, fn, *a):
            # each leg's device objects (programs, graphs, statevectors) are released
            # before the next one starts
            line[key] = fn(*a)
            gc.collect()

        leg("qft", qft_leg)
        if not args.no_sweep:
            leg("fusion_sweep", fusion_sweep_leg, n, args.depth)
            leg("tensor_path", tensor_leg, n, args.depth, line["fusion_sweep"])
        leg("sampling", sampling_leg, n, args.depth)
        leg("circuit_batch", circuit_batch_leg)
        leg("trajectories", trajectory_leg)
        leg("serving", serving_leg, args.serve_requests)
        if not args.no_largest:
            leg("largest_fit", largest_leg, threads)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
