"""Autotuner: device timings of fused-gate passes, the roofline fit of the
reference's hardware profiler refitted to include the tensor pipe, and the
choice of fusion width (and tensor-core use) for a circuit.

The reference's profiler (src/profile.rs:229-352, fit at :137-183 and
:361-410) sweeps gates across arithmetic intensities, fits a two-segment
roofline GFLOP/s = min(bw_slope * AI, peak) and hands the crossover
AI = peak / bw_slope to the hardware-adaptive cost model
(src/cost_model.rs:120-275).  Here:

  * ``measure_profile`` sweeps dense k-qubit gates (AI = 2^(k+1) scalars per
    amplitude, the same AI definition, gate.rs:261-272) on the CUDA-core path
    and fits the roofline the same way (slope = median of GFLOP/s / AI over the
    lower half of the sweep, peak = the largest GFLOP/s);
  * for complex64 it also times the split-BF16 tensor-core path on k = 5, 6 and
    records its effective ceiling as ``tensor_gflops_s`` with
    ``tensor_min_k = 5``, so ``HardwareProfile.crossover_for(k)`` gives the
    tensor-pipe crossover for wide gates;
  * ``choose_fusion`` fuses the circuit at every width k with the native
    planner and predicts its time from the measured per-pass times (scaled by
    2^(n - n_profile), the passes being memory-bound), then returns the width
    and engine with the least predicted time;
  * ``tune_trajectories`` times the batched-trajectory kernel of a noisy
    circuit at each fusion width and launch shape (threads per CTA, CTAs in
    flight) and returns the fastest;
  * ``tune_kernels`` times, for every class of dense k <= 4 gates with targets
    below qubit 5 (precision, k, the set of such targets), the register kernel
    and the tile kernel at 2048 and 4096 amplitudes a tile, and routes each
    class to its fastest (``set_kernel_choice``); the
    choices go into ``HardwareProfile.kernel_choices`` for later processes.

Command line:

    python -m cast_simulator_b200.autotune gate --k 6 --n 26 --mode tc [--low]
    python -m cast_simulator_b200.autotune profile --n 26 --precision f32 [--out prof.json]
    python -m cast_simulator_b200.autotune choose --n 30 --depth 20 --precision f32
    python -m cast_simulator_b200.autotune choose --circuit qft --n 30 --precision f64
    python -m cast_simulator_b200.autotune traj --n 16 --depth 30
    python -m cast_simulator_b200.autotune kernels --n 26 [--profile prof.json]
"""
from __future__ import annotations

import argparse
import json
import math
from dataclasses import dataclass, field

import numpy as np

from .fusion import FusionConfig, HardwareProfile, optimize_native

# CUDA-core FP64 / FP32, split-BF16 tensor cores (complex64), and the sparse
# (CSR) kernels that gates with k >= 5 and at most 2^k / 4 nonzeros a row take
MODES = ("f64", "f32", "tc", "sf64", "sf32")
TENSOR_KS = (5, 6)
SPARSE_KS = (5, 6, 7)


def haar(k: int, rng: np.random.Generator) -> np.ndarray:
    d = 1 << k
    z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def monomial(k: int, rng: np.random.Generator) -> np.ndarray:
    """A permutation with unit phases (one nonzero a row), the shape of fused
    CX / phase blocks."""
    d = 1 << k
    m = np.zeros((d, d), dtype=complex)
    m[np.arange(d), rng.permutation(d)] = np.exp(2j * np.pi * rng.random(d))
    return m


def is_sparse(matrix: np.ndarray, ztol: float = 1e-12) -> bool:
    """Whether a gate runs on the sparse kernels: k >= 5 and at most 2^k / 4
    nonzeros a row after the generator's snapping (|entry| < ztol / 2^k is zero)."""
    d = matrix.shape[0]
    k = d.bit_length() - 1
    return k >= 5 and int((np.abs(matrix) >= ztol / d).sum()) * 4 <= d * d


def dense_ai(k: int) -> float:
    """Arithmetic intensity of a dense k-qubit gate: scalar nonzeros / 2^k."""
    return 2.0 * (1 << k)


def time_gate(n: int, k: int, mode: str, low: bool = False, reps: int = 5, seed: int = 1) -> float:
    """Seconds for one in-place application of a Haar-random k-qubit gate to a
    2^n statevector (best of ``reps`` after one warm-up), timed with CUDA events
    on the launching stream.  Targets are the top k qubits, or the bottom k when
    ``low``."""
    from .cuda import CudaPrecision, CudaStatevector
    from .simulator import Event, GateProgram, Stream

    if mode not in MODES:
        raise ValueError(f"mode must be one of {MODES}")
    if mode.startswith("s") and k < 5:
        raise ValueError("the sparse kernels take gates of 5 or more qubits")
    prec = CudaPrecision.F64 if mode in ("f64", "sf64") else CudaPrecision.F32
    q = tuple(range(k)) if low else tuple(range(n - k, n))
    prog = GateProgram(prec, n, 1e-12, 1e-12, split_precision=(mode == "tc"))
    rng = np.random.default_rng(seed)
    prog.add(monomial(k, rng) if mode.startswith("s") else haar(k, rng), q)
    sv = CudaStatevector(n, prec)
    sv.zero()
    st = Stream()
    e0, e1 = Event(), Event()
    best = math.inf
    for i in range(reps + 1):
        e0.record(st)
        prog.run(sv, st, use_graph=False)
        e1.record(st)
        e1.sync()
        if i:
            best = min(best, e1.elapsed_s(e0))
    return best


@dataclass
class Probe:
    k: int
    mode: str
    ai: float
    seconds: float
    gflops_s: float
    gib_s: float


def probe(n: int, k: int, mode: str, reps: int = 3) -> Probe:
    t = time_gate(n, k, mode, reps=reps)
    scalar = 8 if mode in ("f64", "sf64") else 4
    sv_bytes = (1 << n) * 2 * scalar
    ai = dense_ai(k)
    return Probe(k, mode, ai, t, ai * (1 << n) * 2.0 / t / 1e9, 2.0 * sv_bytes / t / (1 << 30))


def fit_roofline(probes: list[Probe]) -> tuple[float, float, float]:
    """(bw_slope, peak_gflops, crossover_ai) as profile.rs:137-162: the slope
    is the median GFLOP/s / AI over the lower half of the sweep (sorted by AI),
    the peak the largest observed GFLOP/s."""
    if not probes:
        raise ValueError("fit_roofline needs at least one probe")
    sweep = sorted(probes, key=lambda p: p.ai)
    lower = sweep[: (len(sweep) + 1) // 2]
    ratios = sorted(p.gflops_s / p.ai for p in lower)
    slope = ratios[len(ratios) // 2]
    peak = max(p.gflops_s for p in sweep)
    return slope, peak, (peak / slope if slope > 0 else math.inf)


def roofline_r2(probes: list[Probe], slope: float, peak: float) -> float:
    """Coefficient of determination of min(slope * AI, peak) (profile.rs:164-183)."""
    g = np.array([p.gflops_s for p in probes])
    pred = np.array([min(slope * p.ai, peak) for p in probes])
    ss_tot = float(((g - g.mean()) ** 2).sum())
    return 1.0 if ss_tot < 1e-30 else 1.0 - float(((g - pred) ** 2).sum()) / ss_tot


def profile_from_probes(probes: list[Probe], precision: str, n: int,
                        tensor: list[Probe] | None = None) -> HardwareProfile:
    """HardwareProfile from a CUDA-core sweep (and, for complex64, the tensor
    probes): peak bandwidth and GFLOP/s are the largest observed, the slope and
    crossover come from ``fit_roofline``; the tensor ceiling is the largest
    effective GFLOP/s of the tensor probes."""
    slope, peak, xo = fit_roofline(probes)
    prof = HardwareProfile(
        peak_bw_gib_s=max(p.gib_s for p in probes), peak_gflops_s=peak, bw_slope=slope,
        crossover_ai=xo,
        config={"device": "cuda", "precision": precision, "n_qubits": n,
                "r2": roofline_r2(probes, slope, peak)},
        raw=[p.__dict__ for p in probes + (tensor or [])])
    if tensor:
        prof.tensor_gflops_s = max(p.gflops_s for p in tensor)
        prof.tensor_min_k = min(p.k for p in tensor)
    return prof


def measure_profile(n: int = 26, precision: str = "f32", ks=range(1, 8), reps: int = 3) -> HardwareProfile:
    """Sweep dense gates k = 1..7 on the CUDA-core path (and k = 5, 6 on the
    tensor cores for complex64) and fit the profile."""
    probes = [probe(n, k, precision, reps) for k in ks]
    tensor = [probe(n, k, "tc", reps) for k in TENSOR_KS] if precision == "f32" else None
    return profile_from_probes(probes, precision, n, tensor)


@dataclass
class PassTable:
    """Measured seconds per pass, keyed by (k, mode), at ``n_qubits``."""

    n_qubits: int
    seconds: dict = field(default_factory=dict)

    def predict(self, k: int, mode: str, n: int) -> float:
        key = (k, mode)
        if key not in self.seconds:
            raise KeyError(f"no measured pass time for k={k} mode={mode}")
        return self.seconds[key] * 2.0 ** (n - self.n_qubits)


def measure_pass_table(n: int, precision: str, ks=range(1, 8), tensor: bool = True,
                       reps: int = 3, sparse: bool = True) -> PassTable:
    tab = PassTable(n)
    for k in ks:
        tab.seconds[(k, precision)] = time_gate(n, k, precision, reps=reps)
    if tensor and precision == "f32":
        for k in TENSOR_KS:
            tab.seconds[(k, "tc")] = time_gate(n, k, "tc", reps=reps)
    if sparse:
        for k in SPARSE_KS:
            if k in ks:
                tab.seconds[(k, "s" + precision)] = time_gate(n, k, "s" + precision, reps=reps)
    return tab


def engine_for(k: int, precision: str, split: bool, sparse: bool = False) -> str:
    """The kernel family a fused k-qubit gate runs on in a program: the sparse
    kernels for sparse gates of 5 or more qubits (in either precision mode),
    else the tensor cores for 5- and 6-qubit gates of split-precision complex64
    programs, else the CUDA-core kernels."""
    if sparse and k in SPARSE_KS:
        return "s" + precision
    return "tc" if split and precision == "f32" and k in TENSOR_KS else precision


@dataclass
class Choice:
    fusion_k: int
    split_precision: bool
    predicted_s: float
    candidates: list


def choose_fusion(n: int, gates, precision: str, table: PassTable, ks=range(2, 7),
                  allow_tensor: bool = True) -> Choice:
    """Fuse ``gates`` at each width in ``ks`` (size-only cost, the reference's
    default) and predict the circuit time from ``table``; returns the width and
    engine (CUDA cores, or tensor cores for 5- and 6-qubit gates) with the least
    predicted time.  Each fused gate is priced at the pass time of the kernel
    family the library routes it to (``simulator.gate_engine``): sparse gates at
    the table's "sf64" / "sf32" entries, split-precision tensor gates at "tc"."""
    from .cuda import CudaPrecision
    from .simulator import gate_engine

    prec = CudaPrecision.F64 if precision == "f64" else CudaPrecision.F32
    mode_of = {"sparse": "s" + precision, "sparse_tile": "s" + precision, "tensor": "tc"}
    cands = []
    splits = (False, True) if (allow_tensor and precision == "f32") else (False,)
    for k in ks:
        fused = optimize_native(n, gates, FusionConfig.size_only(k)).gates()
        for split in splits:
            # the library's own routing decides each gate's kernel family
            t = sum(table.predict(g.n_qubits(),
                                  mode_of.get(gate_engine(g.matrix(), g.qubits(), n, prec, split),
                                              precision), n)
                    for g in fused)
            cands.append({"fusion_k": k, "split_precision": split, "fused_gates": len(fused),
                          "predicted_s": t})
    best = min(cands, key=lambda c: c["predicted_s"])
    return Choice(best["fusion_k"], best["split_precision"], best["predicted_s"], cands)


@dataclass
class TrajChoice:
    fusion_k: int
    threads: int
    max_ctas: int
    traj_per_s: float
    candidates: list


def tune_trajectories(circuit, n_traj: int = 4096, ks=(2, 3, 4), threads=(0, 512, 1024),
                      ctas=(0,), reps: int = 2, seed: int = 1) -> TrajChoice:
    """Trajectories per second of ``circuit`` for every fusion width in ``ks``
    and launch shape in ``threads`` x ``ctas`` (0 = the kernel's own choice by
    state size), best of ``reps`` graph replays after one warm-up; returns the
    fastest."""
    import time

    from .simulator import Stream
    from .trajectory import TrajectoryProgram

    st = Stream()
    cands = []
    for k in ks:
        prog = TrajectoryProgram(circuit, k)
        for th in threads:
            for c in ctas:
                prog.set_launch(th, c)
                prog.run(n_traj, seed, st)
                best = math.inf
                for r in range(reps):
                    t0 = time.perf_counter()
                    prog.run(n_traj, seed + 1 + r, st)
                    best = min(best, time.perf_counter() - t0)
                cands.append({"fusion_k": k, "threads": th, "max_ctas": c,
                              "traj_per_s": n_traj / best})
    top = max(cands, key=lambda c: c["traj_per_s"])
    return TrajChoice(top["fusion_k"], top["threads"], top["max_ctas"], top["traj_per_s"], cands)


# (engine, tile bits) candidates for the low-target classes
KERNEL_CANDIDATES = (("register", 0), ("tile", 11), ("tile", 12))


def kernel_classes(ks=range(1, 5)):
    """Every (k, low_mask) class of dense gates with at least one target below
    qubit 5: low_mask is that set of targets as bits."""
    return [(k, m) for k in ks for m in range(1, 32) if bin(m).count("1") <= k]


def class_targets(n: int, k: int, low_mask: int) -> tuple:
    """The representative target set of a class: its low targets, the rest at
    the top, the middle and qubit 8 of an n-qubit register."""
    lows = [b for b in range(5) if (low_mask >> b) & 1]
    return tuple(sorted(lows + [n - 1, n // 2, 8][:k - len(lows)]))


def _time_targets(n: int, prec, q: tuple, reps: int, sv, st, rng) -> float:
    from .simulator import Event, GateProgram

    prog = GateProgram(prec, n, 1e-12, 1e-12)
    prog.add(haar(len(q), rng), q)
    e0, e1 = Event(), Event()
    best = math.inf
    for i in range(reps + 1):
        e0.record(st)
        prog.run(sv, st, use_graph=False)
        e1.record(st)
        e1.sync()
        if i:
            best = min(best, e1.elapsed_s(e0))
    return best


def tune_kernels(n: int = 26, precisions=("f64", "f32"), ks=range(1, 5), reps: int = 5,
                 apply: bool = True, seed: int = 7, margin: float = 0.02) -> list[dict]:
    """Time every candidate kernel on every low-target class (best of ``reps``
    launches of a Haar-random gate on the class's representative targets) and
    return one record per class: its winner, the built-in rule's choice and
    each candidate's milliseconds.  A tile kernel wins only when it beats the
    register kernel by more than ``margin`` (the launch-to-launch spread).  With
    ``apply`` the winners are routed process-wide, else every class goes back to
    the built-in rule."""
    from .cuda import CudaPrecision, CudaStatevector
    from .simulator import Stream, gate_engine, set_kernel_choice

    rng = np.random.default_rng(seed)
    st = Stream()
    out = []
    for pname in precisions:
        prec = CudaPrecision.F64 if pname == "f64" else CudaPrecision.F32
        sv = CudaStatevector(n, prec)
        sv.zero()
        for k, mask in kernel_classes(ks):
            q = class_targets(n, k, mask)
            set_kernel_choice(prec, k, mask, None)
            builtin = gate_engine(haar(k, rng), q, n, prec)
            ms = {}
            for eng, tb in KERNEL_CANDIDATES:
                set_kernel_choice(prec, k, mask, eng, tb)
                ms[f"{eng}{tb or ''}"] = 1e3 * _time_targets(n, prec, q, reps, sv, st, rng)
            (eng, tb), best = min(((c, ms[f"{c[0]}{c[1] or ''}"]) for c in KERNEL_CANDIDATES),
                                  key=lambda x: x[1])
            if best > ms["register"] * (1.0 - margin):
                eng, tb = "register", 0
            set_kernel_choice(prec, k, mask, eng if apply else None, tb if apply else 0)
            out.append({"precision": pname, "k": k, "low_mask": mask, "targets": list(q),
                        "engine": eng, "tile_bits": tb, "builtin": builtin, "ms": ms})
        del sv
    return out


def cxx_table(choices) -> str:
    """The built-in routing table of the gate library (gate_kernels.cu,
    kDefaultChoice) from ``tune_kernels`` records of both precisions: per
    precision and k a 32-character row indexed by the low-target mask, 'r' the
    register kernel, 'a' / 'b' the tile kernel with 2048 / 4096 amplitudes."""
    code = {("register", 0): "r", ("tile", 11): "a", ("tile", 12): "b"}
    tab = {(c["precision"], c["k"], c["low_mask"]): code[(c["engine"], c["tile_bits"])]
           for c in choices}
    lines = []
    for p in ("f32", "f64"):
        rows = ['"' + "".join(tab.get((p, k, m), "-") for m in range(32)) + '"'
                for k in range(1, 5)]
        lines.append("    {\"\", " + ", ".join(rows) + "},")
    return "\n".join(lines)


def apply_kernel_choices(choices) -> int:
    """Route the classes of ``choices`` (``tune_kernels`` records, or a
    ``HardwareProfile`` holding them) process-wide; returns how many."""
    from .cuda import CudaPrecision
    from .simulator import set_kernel_choice

    if isinstance(choices, HardwareProfile):
        choices = choices.kernel_choices
    for c in choices:
        prec = CudaPrecision.F64 if c["precision"] == "f64" else CudaPrecision.F32
        set_kernel_choice(prec, c["k"], c["low_mask"], c["engine"], c["tile_bits"])
    return len(choices)


def _main(argv=None) -> None:
    ap = argparse.ArgumentParser(prog="python -m cast_simulator_b200.autotune")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("gate", help="time one Haar-random gate application")
    g.add_argument("--k", type=int, required=True)
    g.add_argument("--n", type=int, default=26)
    g.add_argument("--mode", choices=MODES, default="f32")
    g.add_argument("--low", action="store_true", help="targets are qubits 0..k-1")
    g.add_argument("--reps", type=int, default=5)
    p = sub.add_parser("profile", help="roofline profile with the tensor-pipe crossover")
    p.add_argument("--n", type=int, default=26)
    p.add_argument("--precision", choices=("f64", "f32"), default="f32")
    p.add_argument("--out")
    c = sub.add_parser("choose", help="fusion width / engine for a brickwork or QFT-CX circuit")
    c.add_argument("--circuit", choices=("brickwork", "qft"), default="brickwork")
    c.add_argument("--n", type=int, default=30)
    c.add_argument("--depth", type=int, default=20, help="brickwork depth")
    c.add_argument("--precision", choices=("f64", "f32"), default="f32")
    c.add_argument("--profile-n", type=int, default=26)
    t = sub.add_parser("traj", help="fusion width / launch shape for noisy brickwork trajectories")
    t.add_argument("--n", type=int, default=16)
    t.add_argument("--depth", type=int, default=30)
    t.add_argument("--traj", type=int, default=4096)
    t.add_argument("--p", type=float, default=1e-3)
    t.add_argument("--gamma", type=float, default=5e-4)
    kk = sub.add_parser("kernels", help="register / tile kernel and tile size per low-target class")
    kk.add_argument("--n", type=int, default=26)
    kk.add_argument("--precision", choices=("f64", "f32", "both"), default="both")
    kk.add_argument("--reps", type=int, default=5)
    kk.add_argument("--profile", help="profile JSON to store the choices in (created if absent)")
    kk.add_argument("--cxx-table", action="store_true",
                    help="print the winners as the library's built-in routing table")
    a = ap.parse_args(argv)
    if a.cmd == "kernels":
        import os

        precs = ("f64", "f32") if a.precision == "both" else (a.precision,)
        ch = tune_kernels(a.n, precs, reps=a.reps)
        if a.profile:
            prof = (HardwareProfile.load(a.profile) if os.path.exists(a.profile)
                    else HardwareProfile(0.0, 0.0, 0.0, math.inf))
            keep = [c for c in prof.kernel_choices if c["precision"] not in precs]
            prof.kernel_choices = keep + ch
            prof.save(a.profile)
        print(cxx_table(ch) if a.cxx_table else json.dumps({"n": a.n, "choices": ch}))
    elif a.cmd == "traj":
        from .types import QuantumCircuit

        circ = QuantumCircuit.brickwork(a.n, a.depth, 31337, depolarizing=a.p, damping=a.gamma)
        ch = tune_trajectories(circ, a.traj)
        print(json.dumps({"fusion_k": ch.fusion_k, "threads": ch.threads, "max_ctas": ch.max_ctas,
                          "traj_per_s": ch.traj_per_s, "candidates": ch.candidates}))
    elif a.cmd == "gate":
        t = time_gate(a.n, a.k, a.mode, a.low, a.reps)
        b = 2 * (1 << a.n) * (16 if a.mode in ("f64", "sf64") else 8)
        print(json.dumps({"k": a.k, "n": a.n, "mode": a.mode, "low_targets": a.low,
                          "ms": t * 1e3, "gb_s": b / t / 1e9}))
    elif a.cmd == "profile":
        prof = measure_profile(a.n, a.precision)
        if a.out:
            prof.save(a.out)
        d = dict(prof.__dict__)
        d.pop("raw")
        d["crossover_tensor_ai"] = prof.crossover_for(prof.tensor_min_k) if prof.tensor_min_k else None
        print(json.dumps(d))
    else:
        from .types import QuantumCircuit

        circ = (QuantumCircuit.brickwork(a.n, a.depth, 2024) if a.circuit == "brickwork"
                else QuantumCircuit.qft_cx(a.n))
        tab = measure_pass_table(a.profile_n, a.precision)
        ch = choose_fusion(a.n, circ.gates(), a.precision, tab)
        print(json.dumps({"fusion_k": ch.fusion_k, "split_precision": ch.split_precision,
                          "predicted_ms": ch.predicted_s * 1e3, "candidates": ch.candidates}))


if __name__ == "__main__":
    _main()
