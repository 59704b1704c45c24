"""Simulator API: host-side mirror of src/simulator/{mod,bench,measure}.rs.

``Simulator`` (mod.rs:446-547) owns the precision / tolerance spec and runs a
``CircuitGraph``: ``simulate`` returns a ``QuantumState`` for the state-vector
or density-matrix representation (mod.rs:523-547, prepare_gates at
mod.rs:586-613); ``bench`` compiles once and times repeated executions with
device events (bench.rs:136-167, timing.rs:88-130).  Gates go to the GPU as a
``GateProgram`` (include/cast_b200.h), replayed as a CUDA graph.
"""
from __future__ import annotations

import ctypes as C
import enum
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .cuda import CudaKernelGenSpec, CudaPrecision, CudaStatevector
from .fusion import CircuitGraph


class Representation(enum.Enum):
    StateVector = 0
    DensityMatrix = 1


class Stream:
    """An owned CUDA stream.  Non-blocking by default (it does not synchronise
    with the legacy default stream, so a graph capture on it cannot be
    invalidated by other threads' stream-0 work); ``blocking=True`` gives the
    reference's CU_STREAM_DEFAULT kind (cast_cuda_stream_create)."""

    def __init__(self, blocking: bool = False, priority: int | None = None):
        """priority: a non-blocking stream with this scheduling priority (lower is
        more urgent, clamped into the device's range; see
        cast_b200_stream_create_priority)."""
        eb = L.errbuf()
        if priority is not None:
            self.handle = L.check_ptr(L.lib().cast_b200_stream_create_priority(int(priority), eb,
                                                                               L.ERR_LEN), eb, "stream")
            return
        fn = L.lib().cast_cuda_stream_create if blocking else L.lib().cast_b200_stream_create_nonblocking
        self.handle = L.check_ptr(fn(eb, L.ERR_LEN), eb, "stream")

    def sync(self):
        eb = L.errbuf()
        L.check(L.lib().cast_cuda_stream_sync(self.handle, eb, L.ERR_LEN), eb, "stream sync")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().cast_cuda_stream_destroy(h)
            except Exception:
                pass


class Event:
    def __init__(self):
        eb = L.errbuf()
        self.handle = L.check_ptr(L.lib().cast_cuda_event_create(eb, L.ERR_LEN), eb, "event")

    def record(self, stream):
        """Record on a Stream or on a raw stream handle."""
        h = stream.handle if isinstance(stream, Stream) else stream
        eb = L.errbuf()
        L.check(L.lib().cast_cuda_event_record(self.handle, h, eb, L.ERR_LEN), eb, "record")

    def elapsed_s(self, start: "Event") -> float:
        eb = L.errbuf()
        ms = C.c_float()
        L.check(L.lib().cast_cuda_event_elapsed_ms(start.handle, self.handle, C.byref(ms), eb,
                                                   L.ERR_LEN), eb, "elapsed")
        return ms.value * 1e-3

    def sync(self):
        eb = L.errbuf()
        L.check(L.lib().cast_cuda_event_synchronize(self.handle, eb, L.ERR_LEN), eb, "event sync")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().cast_cuda_event_destroy(h)
            except Exception:
                pass


class GateProgram:
    """Ordered gates for one statevector size, uploaded once (cast_b200_program_*)."""

    def __init__(self, precision: CudaPrecision, n_qubits: int, ztol: float, otol: float,
                 split_precision: bool = False):
        eb = L.errbuf()
        self.handle = L.check_ptr(
            L.lib().cast_b200_program_create(int(precision), n_qubits, ztol, otol, eb, L.ERR_LEN), eb,
            "program_create")
        if split_precision:
            L.check(L.lib().cast_b200_program_set_split_precision(self.handle, 1, eb, L.ERR_LEN), eb,
                    "set_split_precision")
        self.n_qubits = n_qubits
        self.precision = CudaPrecision(precision)
        self.gate_sizes: list[int] = []

    def add(self, matrix: np.ndarray, qubits) -> None:
        m = np.ascontiguousarray(matrix, dtype=np.complex128)
        q = np.ascontiguousarray(qubits, dtype=np.uint32)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_program_add_gate(
            self.handle, m.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)),
            q.ctypes.data_as(L.c_u32p), q.size, eb, L.ERR_LEN), eb, "program_add_gate")
        self.gate_sizes.append(int(q.size))

    def __len__(self):
        return int(L.lib().cast_b200_program_num_gates(self.handle))

    def run(self, sv: CudaStatevector, stream: Stream | None = None, use_graph: bool = True) -> None:
        if sv.n_qubits() != self.n_qubits or sv.precision() != self.precision:
            raise ValueError("statevector does not match the program")
        eb = L.errbuf()
        L.check(L.lib().cast_b200_program_run(self.handle, sv.dptr, stream.handle if stream else None,
                                              int(use_graph), eb, L.ERR_LEN), eb, "program_run")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().cast_b200_program_destroy(h)
            except Exception:
                pass


def tensor_status() -> int:
    """Reads and clears the tensor-core kernel's error word: 0 when every
    bounded wait inside every tensor-core launch since the last call completed."""
    eb = L.errbuf()
    out = C.c_uint32()
    L.check(L.lib().cast_b200_tensor_status(C.byref(out), eb, L.ERR_LEN), eb, "tensor_status")
    return out.value


ENGINES = ("register", "tile", "staged", "sparse", "sparse_tile", "tensor")


def gate_engine(matrix: np.ndarray, qubits, n_qubits: int, precision: CudaPrecision,
                split_precision: bool = False, ztol: float = 1e-12, otol: float = 1e-12) -> str:
    """The kernel family a gate would run on in a gate program of ``n_qubits``
    (one of ``ENGINES``), decided by the library exactly as a launch decides
    it, without touching the device."""
    from .types import _canonicalize

    m, qs = _canonicalize(np.asarray(matrix, dtype=np.complex128), list(qubits))
    m = np.ascontiguousarray(m)
    q = np.ascontiguousarray(qs, dtype=np.uint32)
    eb = L.errbuf()
    e = L.lib().cast_b200_gate_engine(int(precision), n_qubits,
                                      m.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)),
                                      q.ctypes.data_as(L.c_u32p), q.size, ztol, otol,
                                      int(split_precision), eb, L.ERR_LEN)
    if e < 0:
        raise RuntimeError(f"gate_engine failed: {eb.value.decode()}")
    return ENGINES[e]


def set_kernel_choice(precision: CudaPrecision, k: int, low_mask: int, engine: str | None,
                      tile_bits: int = 0) -> None:
    """Route one class of dense gates (k <= 4 qubits, the targets below qubit 5
    forming ``low_mask``) to the ``"register"`` or ``"tile"`` kernel, with
    2^``tile_bits`` amplitudes a tile (11, 12, or 0 for the built-in size);
    ``engine=None`` restores the built-in rule.  Process-wide, for launches after
    the call."""
    code = {None: -1, "register": 0, "tile": 1}[engine]
    eb = L.errbuf()
    L.check(L.lib().cast_b200_set_kernel_choice(int(precision), k, low_mask, code, tile_bits, eb,
                                                L.ERR_LEN), eb)


def inner_product(a: CudaStatevector, b: CudaStatevector, stream: Stream | None = None) -> complex:
    if a.n_qubits() != b.n_qubits() or a.precision() != b.precision():
        raise ValueError("statevector size/precision mismatch")
    re, im = C.c_double(), C.c_double()
    eb = L.errbuf()
    L.check(L.lib().cast_b200_inner_product(a.dptr, b.dptr, a.n_qubits(), int(a.precision()),
                                            C.byref(re), C.byref(im),
                                            stream.handle if stream else None, eb, L.ERR_LEN), eb,
            "inner_product")
    return complex(re.value, im.value)


def qubit_populations(sv: CudaStatevector, stream: Stream | None = None) -> tuple[np.ndarray, float]:
    """(P(q=1) for every qubit, norm^2), one FP64 device pass."""
    out = np.zeros(sv.n_qubits())
    nrm = C.c_double()
    eb = L.errbuf()
    L.check(L.lib().cast_b200_qubit_populations(sv.dptr, sv.n_qubits(), int(sv.precision()),
                                                out.ctypes.data_as(L.c_dp), C.byref(nrm),
                                                stream.handle if stream else None, eb, L.ERR_LEN),
            eb, "qubit_populations")
    return out, nrm.value


def marginal_probabilities(sv: CudaStatevector, measured, stream: Stream | None = None) -> np.ndarray:
    q = np.ascontiguousarray(measured, dtype=np.uint32)
    out = np.zeros(1 << q.size)
    eb = L.errbuf()
    L.check(L.lib().cast_b200_marginal_probabilities(
        sv.dptr, sv.n_qubits(), int(sv.precision()), q.ctypes.data_as(L.c_u32p), q.size,
        out.ctypes.data_as(L.c_dp), stream.handle if stream else None, eb, L.ERR_LEN), eb,
        "marginal_probabilities")
    return out


class CircuitBatch:
    """Many small circuits run in one persistent launch (cast_b200_batch_*): one
    CTA a circuit on its own device statevector, each circuit's <Z_q> reduced in
    FP64 on the device.  ``add`` takes a gate list (objects with ``matrix()`` /
    ``qubits()``, at most 4 qubits a gate - fuse with size_max <= 4) or a native
    fused circuit; ``run`` executes every circuit added since the last
    ``clear`` and returns their <Z> vectors in the order they were added."""

    def __init__(self):
        eb = L.errbuf()
        self.handle = L.check_ptr(L.lib().cast_b200_batch_create(eb, L.ERR_LEN), eb, "batch_create")
        self._sizes: list[int] = []

    def add(self, sv: CudaStatevector, gates, init_zero: bool = True, ztol: float | None = None,
            otol: float | None = None) -> int:
        """Append a circuit acting on `sv`; returns its index in the batch."""
        f64 = sv.precision() == CudaPrecision.F64
        zt = ztol if ztol is not None else (1e-12 if f64 else 1e-6)
        ot = otol if otol is not None else (1e-12 if f64 else 1e-6)
        eb = L.errbuf()
        if hasattr(gates, "handle"):  # a native fused circuit
            rc = L.lib().cast_b200_batch_add_fused(self.handle, sv.dptr, sv.n_qubits(),
                                                   int(sv.precision()), gates.handle, int(init_zero),
                                                   zt, ot, eb, L.ERR_LEN)
        else:
            gates = list(gates)
            ks = np.array([len(g.qubits()) for g in gates], dtype=np.uint32)
            qs = np.array([q for g in gates for q in g.qubits()], dtype=np.uint32)
            ms = (np.concatenate([np.ascontiguousarray(g.matrix(), dtype=np.complex128).reshape(-1)
                                  for g in gates]) if gates else np.zeros(1, dtype=np.complex128))
            rc = L.lib().cast_b200_batch_add(self.handle, sv.dptr, sv.n_qubits(), int(sv.precision()),
                                             len(gates), ks.ctypes.data_as(L.c_u32p),
                                             qs.ctypes.data_as(L.c_u32p),
                                             ms.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)),
                                             int(init_zero), zt, ot, eb, L.ERR_LEN)
        L.check(rc, eb, "batch_add")
        self._sizes.append(sv.n_qubits())
        return len(self._sizes) - 1

    def __len__(self):
        return len(self._sizes)

    def run(self, stream: Stream | None = None) -> list[np.ndarray]:
        out = np.zeros(max(1, sum(self._sizes)))
        eb = L.errbuf()
        L.check(L.lib().cast_b200_batch_run(self.handle, out.ctypes.data_as(L.c_dp),
                                            stream.handle if stream else None, eb, L.ERR_LEN),
                eb, "batch_run")
        res, at = [], 0
        for n in self._sizes:
            res.append(out[at:at + n].copy())
            at += n
        return res

    def clear(self) -> None:
        L.lib().cast_b200_batch_clear(self.handle)
        self._sizes.clear()

    def __del__(self):
        try:
            L.lib().cast_b200_batch_destroy(self.handle)
        except Exception:
            pass


def sample(sv: CudaStatevector, n_shots: int, seed: int = 0, measured=None,
           stream: Stream | None = None, uniforms=None, out: np.ndarray | None = None) -> np.ndarray:
    """Shot keys sampled on the device from |a_i|^2 (cast_b200_sample): the
    sampled basis indices, or with `measured` their bits at those qubits packed
    into bits 0..m-1 (the reference's compress_bits), in ascending order of the
    sampled index.  `uniforms` (sorted, in [0, 1), one a shot) replaces the
    device's Philox draws (cast_b200_sample_at).  `out` (a contiguous uint64
    array of n_shots, e.g. a reused page-locked buffer) receives the keys and is
    returned; by default a new array is allocated."""
    q = np.ascontiguousarray([] if measured is None else list(measured), dtype=np.uint32)
    if out is None:
        out = np.empty(n_shots, dtype=np.uint64)
    elif out.dtype != np.uint64 or out.size != n_shots or not out.flags["C_CONTIGUOUS"]:
        raise ValueError("out must be a contiguous uint64 array of n_shots")
    eb = L.errbuf()
    qp = q.ctypes.data_as(L.c_u32p) if q.size else None
    h = stream.handle if stream else None
    if uniforms is None:
        rc = L.lib().cast_b200_sample(sv.dptr, sv.n_qubits(), int(sv.precision()), n_shots,
                                      seed & ((1 << 64) - 1), qp, q.size,
                                      out.ctypes.data_as(L.c_u64p), h, eb, L.ERR_LEN)
    else:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        if u.size != n_shots:
            raise ValueError("one uniform a shot")
        rc = L.lib().cast_b200_sample_at(sv.dptr, sv.n_qubits(), int(sv.precision()),
                                         u.ctypes.data_as(L.c_dp), n_shots, qp, q.size,
                                         out.ctypes.data_as(L.c_u64p), h, eb, L.ERR_LEN)
    L.check(rc, eb, "sample")
    return out


def sample_histogram(sv: CudaStatevector, n_shots: int, seed: int = 0, measured=None,
                     stream: Stream | None = None) -> dict:
    """{outcome: count} over the measured qubits (all qubits when None): the
    reference's batch_sample result (src/simulator/measure.rs:49-76), drawn on
    the device without downloading the statevector."""
    keys = sample(sv, n_shots, seed, measured, stream)
    vals, counts = np.unique(keys, return_counts=True)
    return {int(k): int(c) for k, c in zip(vals, counts)}


def prepare_gates(graph: CircuitGraph, n_physical: int, repr_: Representation):
    """mod.rs:586-613: SV needs unitary gates; DM lifts each gate to a
    superoperator on 2n virtual qubits."""
    gates = graph.gates_in_row_order()
    if repr_ == Representation.StateVector:
        for i, g in enumerate(gates):
            if not g.is_unitary():
                raise ValueError(
                    f"gate index {i} is non-unitary; Representation.StateVector requires unitary "
                    "gates (use DensityMatrix or sample_trajectory for noisy circuits)")
        return gates, n_physical
    return [g.to_density_matrix_gate(n_physical) for g in gates], 2 * n_physical


class QuantumState:
    """mod.rs:320-414 (CUDA inspection methods)."""

    def __init__(self, sv: CudaStatevector, n_physical: int, repr_: Representation):
        self.sv, self._n, self._repr = sv, n_physical, repr_

    def n_qubits(self) -> int:
        return self._n

    def is_pure(self) -> bool:
        return self._repr == Representation.StateVector

    def download_amplitudes(self) -> np.ndarray:
        return self.sv.download()

    def populations(self) -> np.ndarray:
        if self.is_pure():
            return np.abs(self.sv.download()) ** 2
        out = np.zeros(1 << self._n)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_dm_populations(self.sv.dptr, self._n, int(self.sv.precision()),
                                                 out.ctypes.data_as(L.c_dp), None, eb, L.ERR_LEN),
                eb, "dm_populations")
        return out

    def trace(self) -> float:
        if self.is_pure():
            return self.sv.norm_squared()
        return float(self.populations().sum())

    def sample(self, n_shots: int, measured=None, seed: int = 0) -> dict:
        """Histogram {outcome: count} of n_shots measurements of the measured
        qubits (all when None), drawn on the device (pure states)."""
        if not self.is_pure():
            raise ValueError("sampling is for statevectors; use the trajectory sampler for "
                             "noisy circuits")
        return sample_histogram(self.sv, n_shots, seed, measured)

    def expectation_z(self) -> np.ndarray:
        """<Z_q> for every physical qubit (pure states), FP64 on the device."""
        if not self.is_pure():
            p = self.populations()
            idx = np.arange(p.size)
            return np.array([1 - 2 * p[(idx >> q) & 1 == 1].sum() for q in range(self._n)])
        p1, nrm = qubit_populations(self.sv)
        return (nrm - 2 * p1) / nrm


@dataclass
class PhaseTiming:
    """bench.rs:42-110: raw samples of one phase (seconds)."""

    samples_s: list = field(default_factory=list)
    source: str = "gpu_events"

    def mean_s(self):
        return float(np.mean(self.samples_s)) if self.samples_s else 0.0

    def stddev_s(self):
        return float(np.std(self.samples_s, ddof=1)) if len(self.samples_s) > 1 else 0.0

    def min_s(self):
        return float(np.min(self.samples_s)) if self.samples_s else 0.0


@dataclass
class RunTiming:
    compile: PhaseTiming
    exec: PhaseTiming
    n_gates: int
    n_qubits: int


class Simulator:
    """Simulator<Cuda> (mod.rs:446-547)."""

    def __init__(self, spec: CudaKernelGenSpec | None = None, use_graph: bool = True,
                 split_precision: bool = False, reuse_memory: bool = True):
        """split_precision: complex64 gates with 5 or 6 qubits run on the tensor
        cores in split BF16 (about 1e-5 relative error per fused pass).
        reuse_memory: when a returned QuantumState is dropped, its statevector
        allocation is kept (one per qubit count and precision) for the next
        ``simulate`` instead of being freed; ``release_memory`` frees them."""
        self.spec = spec or CudaKernelGenSpec.f64()
        self.use_graph = use_graph
        self.split_precision = split_precision
        self._stream = None
        self.reuse_memory = reuse_memory
        self._free: dict = {}  # (n, precision) -> (dptr, len)

    def _release(self, n, prec, dptr, length) -> bool:
        key = (n, int(prec))
        if not self.reuse_memory or key in self._free:
            return False
        self._free[key] = (dptr, length)
        return True

    def _statevector(self, n: int) -> CudaStatevector:
        hit = self._free.pop((n, int(self.spec.precision)), None)
        if hit is not None:
            return CudaStatevector._adopt(n, self.spec.precision, hit[0], self._release)
        sv = CudaStatevector(n, self.spec.precision)
        sv._release = self._release if self.reuse_memory else None
        return sv

    def release_memory(self) -> None:
        """Free the statevector allocations kept for reuse."""
        for dptr, _ in self._free.values():
            L.lib().cast_cuda_sv_free(dptr)
        self._free.clear()

    def __del__(self):
        try:
            self.release_memory()
        except Exception:
            pass

    @classmethod
    def f64(cls) -> "Simulator":
        return cls(CudaKernelGenSpec.f64())

    @classmethod
    def f32(cls) -> "Simulator":
        return cls(CudaKernelGenSpec.f32())

    @property
    def stream(self) -> Stream:
        if self._stream is None:
            self._stream = Stream()
        return self._stream

    def compile_batch(self, gates, n_sv: int) -> GateProgram:
        prog = GateProgram(self.spec.precision, n_sv, self.spec.ztol, self.spec.otol,
                           self.split_precision and self.spec.precision == CudaPrecision.F32)
        for i, g in enumerate(gates):
            try:
                prog.add(g.matrix(), g.qubits())
            except L.CudaError as e:
                raise L.CudaError(f"generating kernel for gate index {i}: {e}") from e
        return prog

    def simulate(self, graph: CircuitGraph, repr_: Representation = Representation.StateVector,
                 initial: np.ndarray | None = None) -> QuantumState:
        n_phys = graph.n_qubits()
        gates, n_sv = prepare_gates(graph, n_phys, repr_)
        prog = self.compile_batch(gates, n_sv)
        sv = self._statevector(n_sv)
        if initial is None:
            sv.zero(self.stream)
        else:
            sv.upload(initial)
        prog.run(sv, self.stream, self.use_graph)
        self.stream.sync()
        return QuantumState(sv, n_phys, repr_)

    def bench(self, graph: CircuitGraph, repr_: Representation = Representation.StateVector,
              budget_s: float = 1.0, min_iters: int = 3) -> RunTiming:
        """Compile once, then time zero + apply-all on the device until the
        budget is spent (25% of it as warm-up, timing.rs:88-130)."""
        n_phys = graph.n_qubits()
        t0 = time.perf_counter()
        gates, n_sv = prepare_gates(graph, n_phys, repr_)
        prog = self.compile_batch(gates, n_sv)
        comp = PhaseTiming([time.perf_counter() - t0], "wall")
        sv = CudaStatevector(n_sv, self.spec.precision)
        st = self.stream
        e0, e1 = Event(), Event()

        def one():
            sv.zero(st)
            e0.record(st)
            prog.run(sv, st, self.use_graph)
            e1.record(st)
            e1.sync()
            return e1.elapsed_s(e0)

        probe = one()
        n_total = max(min_iters, int(budget_s / max(probe, 1e-6)))
        n_warm = max(1, n_total // 4)
        for _ in range(n_warm):
            one()
        samples = [one() for _ in range(max(min_iters, n_total - n_warm))]
        return RunTiming(comp, PhaseTiming(samples), len(prog), n_sv)
