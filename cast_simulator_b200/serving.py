"""Continuous-batching request loop for circuit simulation on one GPU.

The reference runs one circuit at a time through ``Simulator::simulate`` /
``sample_trajectory`` (src/simulator/mod.rs:523-547, trajectory.rs:104-130);
this engine keeps many requests in flight:

  * requests (a circuit, a precision, optionally a trajectory count) queue in
    arrival order;
  * a dispatcher admits the head of the queue as soon as a slot is free and the
    device-memory budget covers its footprint (16 * 2^n bytes for complex128,
    8 * 2^n for complex64, the trajectory workspace for noisy requests);
    admission never reorders requests;
  * a small pure request (at most ``batch_max_qubits`` qubits) goes to the
    batcher: every small request admitted while the previous batch ran is fused
    by the native planner and executed with the others in ONE persistent launch
    of the circuit-batch kernel (one CTA a circuit, <Z_q> reduced on the device)
    when there are at least ``batch_min`` of them; a smaller batch runs its
    requests one after another on the plain kernels, which take every SM for a
    fraction of a millisecond instead of holding a few SMs for milliseconds in
    the way of the persistent kernels of the large requests;
  * any other admitted request runs on its own CUDA stream in a worker thread:
    its gates are fused by the native planner and uploaded as a gate program
    that is launched on that stream (noisy requests run the persistent
    trajectory kernel from a CUDA graph); work of different requests overlaps on
    the device;
  * when a request finishes, its <Z_q> vector is read back (FP64 device
    reduction), its memory returns to the budget and the next requests are
    admitted - the batch composition changes continuously.

Statevectors are recycled through a per-(qubits, precision) free list, so
steady-state admission does not call cudaMalloc.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .cuda import CudaPrecision, CudaStatevector, cuda_free_memory_bytes
from .fusion import FusionConfig, optimize_native
from .simulator import CircuitBatch, GateProgram, Stream, qubit_populations
from .trajectory import TrajectoryProgram
from .types import QuantumCircuit


@dataclass
class Request:
    circuit: QuantumCircuit
    precision: CudaPrecision = CudaPrecision.F64
    n_traj: int = 0  # 0: pure state-vector simulation
    seed: int = 0
    arrival: float = 0.0  # seconds after the stream starts (run_stream)
    rid: int = -1


@dataclass
class Result:
    rid: int
    z: np.ndarray  # <Z_q> for every qubit (trajectory mean for noisy requests)
    arrival: float
    admitted: float
    finished: float
    n_qubits: int
    precision: CudaPrecision
    n_traj: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_bytes(req: Request, sm_count: int = 148) -> int:
    n = req.circuit.n_qubits()
    if req.n_traj:
        return (8 << n) * min(req.n_traj, sm_count) + 8 * req.n_traj * (n + 1)
    return (16 if req.precision == CudaPrecision.F64 else 8) << n


class _SvPool:
    """Free lists of device statevectors keyed by (qubits, precision)."""

    def __init__(self):
        self._free: dict = collections.defaultdict(list)
        self._lock = threading.Lock()

    def get(self, n: int, prec: CudaPrecision) -> CudaStatevector:
        with self._lock:
            lst = self._free[(n, prec)]
            if lst:
                return lst.pop()
        return CudaStatevector(n, prec)

    def put(self, sv: CudaStatevector) -> None:
        with self._lock:
            self._free[(sv.n_qubits(), sv.precision())].append(sv)

    def drop_all(self) -> int:
        with self._lock:
            n = sum(len(v) for v in self._free.values())
            self._free.clear()
        return n

    def cached_bytes(self) -> int:
        with self._lock:
            return sum(sv.nbytes() for v in self._free.values() for sv in v)


class ServingEngine:
    def __init__(self, max_slots: int = 8, mem_budget_bytes: int | None = None, fusion_k: int = 4,
                 traj_fusion_k: int | None = None, use_graph: bool = False,
                 batch_max_qubits: int = 16, batch_fusion_k: int = 3, max_batch: int = 1024,
                 batch_min: int = 32,
                 split_min_qubits: int = 20, heavy_slots: int = 1, heavy_pure_qubits: int = 22,
                 heavy_noisy_qubits: int = 17, heavy_priority: bool = False):
        """max_slots: requests running at once on the worker streams.
        traj_fusion_k: fusion width of noisy requests' trajectory programs (None:
        3 up to 16 qubits, where the states sit in L1/L2 and the passes are bound
        by instruction issue, 4 above, where fewer passes over HBM win).
        split_min_qubits: complex64 pure requests of at least this many qubits
        run as split-precision programs fused at k = 6 (dense 5- and 6-qubit
        gates on the tensor cores, 1 - |<ref|psi>| ~ 1e-10; 0 turns it off).
        heavy_slots: requests that fill the GPU by themselves (pure requests of
        heavy_pure_qubits or more qubits, noisy ones of heavy_noisy_qubits or
        more) execute on the GPU at most this many at a time: two of them running
        together only interleave, and each finishes later than if they ran one
        after the other.  Only the device phase waits: a heavy request is
        admitted as usual and fuses and builds its program while another one
        runs, and small requests still overlap with it.
        heavy_priority: heavy requests run on a more urgent stream (their thread
        blocks start first when SMs free up), so the small requests around them
        slow them down less.
        batch_max_qubits: pure requests of at most this many qubits run batched
        in the circuit-batch kernel (0 turns batching off); batch_fusion_k: their
        fusion width (<= 4); max_batch: circuits a batch launch takes at most
        (batched requests do not use worker slots); batch_min: the fewest
        circuits the batch kernel is launched for (fewer run on the plain
        kernels in the batcher thread: a batch of one circuit would hold one SM
        for its whole run)."""
        if mem_budget_bytes is None:
            free, _ = cuda_free_memory_bytes()
            mem_budget_bytes = int(free * 0.8)
        if not 0 <= batch_max_qubits <= 20 or not 1 <= batch_fusion_k <= 4:
            raise ValueError("batch_max_qubits must be 0..20 and batch_fusion_k 1..4")
        self.max_slots = max_slots
        self.budget = mem_budget_bytes
        self.fusion_k = fusion_k
        self.traj_fusion_k = traj_fusion_k
        self.use_graph = use_graph
        self.batch_max_qubits = batch_max_qubits
        self.batch_fusion_k = batch_fusion_k
        self.max_batch = max_batch
        self.batch_min = max(1, batch_min)
        self.small_plain_requests = 0
        self.split_min_qubits = split_min_qubits
        self.heavy_slots = heavy_slots
        self.heavy_pure_qubits = heavy_pure_qubits
        self.heavy_noisy_qubits = heavy_noisy_qubits
        self._gpu_heavy = threading.Semaphore(max(1, heavy_slots))
        self.heavy_priority = heavy_priority
        self._bwork: collections.deque = collections.deque()
        self._bcv = threading.Condition()
        self._batched_active = 0
        self.batches_run = 0
        self.batched_requests = 0
        self._pool = _SvPool()
        self._pending: collections.deque = collections.deque()
        self._cv = threading.Condition()
        self._in_use = 0
        self._active = 0
        self._stop = False
        self._t0 = time.perf_counter()
        self._work: collections.deque = collections.deque()
        self._work_cv = threading.Condition()
        self.max_concurrent = 0
        self._workers = [threading.Thread(target=self._worker, daemon=True) for _ in range(max_slots)]
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._batcher = threading.Thread(target=self._batch_loop, daemon=True)
        for t in self._workers:
            t.start()
        self._dispatcher.start()
        self._batcher.start()

    # -- public API
    def now(self) -> float:
        return time.perf_counter() - self._t0

    def submit(self, req: Request) -> Future:
        need = request_bytes(req)
        if need > self.budget:
            raise ValueError(f"request needs {need} bytes, above the device-memory budget {self.budget}")
        fut: Future = Future()
        with self._cv:
            if self._stop:
                raise RuntimeError("the serving engine has been shut down")
            self._pending.append((req, fut, self.now()))
            self._cv.notify_all()
        return fut

    def run_stream(self, requests: list[Request]) -> list[Result]:
        """Submit requests at their arrival offsets (real time) and wait for all."""
        base = self.now()
        futs = []
        for r in sorted(requests, key=lambda x: x.arrival):
            delay = base + r.arrival - self.now()
            if delay > 0:
                time.sleep(delay)
            futs.append(self.submit(r))
        return [f.result() for f in futs]

    def shutdown(self) -> None:
        """Stop admitting: requests already admitted run to completion, requests
        still waiting for admission fail with RuntimeError."""
        with self._cv:
            self._stop = True
            pending = list(self._pending)
            self._pending.clear()
            self._cv.notify_all()
        for _, fut, _ in pending:
            fut.set_exception(RuntimeError("the serving engine was shut down before admission"))
        with self._work_cv:
            self._work_cv.notify_all()
        with self._bcv:
            self._bcv.notify_all()
        self._dispatcher.join(timeout=30)
        for t in self._workers:
            t.join(timeout=30)
        self._batcher.join(timeout=30)
        self._pool.drop_all()

    # -- internals
    def _dispatch(self) -> None:
        while True:
            with self._cv:
                while not self._stop and not self._can_admit_head():
                    self._cv.wait(timeout=0.05)
                if self._stop:
                    return
                req, fut, t_arr = self._pending.popleft()
                need = request_bytes(req)
                self._in_use += need
                batched = self._batchable(req)
                if batched:
                    self._batched_active += 1
                else:
                    self._active += 1
                self.max_concurrent = max(self.max_concurrent, self._active + self._batched_active)
            if batched:
                with self._bcv:
                    self._bwork.append((req, fut, t_arr, need, self.now()))
                    self._bcv.notify()
            else:
                with self._work_cv:
                    self._work.append((req, fut, t_arr, need, self.now()))
                    self._work_cv.notify()

    def _batchable(self, req: Request) -> bool:
        return not req.n_traj and req.circuit.n_qubits() <= self.batch_max_qubits

    def _heavy(self, req: Request) -> bool:
        n = req.circuit.n_qubits()
        return n >= (self.heavy_noisy_qubits if req.n_traj else self.heavy_pure_qubits)

    def _can_admit_head(self) -> bool:
        if not self._pending:
            return False
        head = self._pending[0][0]
        if self._batchable(head):
            if self._batched_active >= self.max_batch:
                return False
        elif self._active >= self.max_slots:
            return False
        need = request_bytes(self._pending[0][0])
        if self._in_use + need > self.budget:
            return False
        if self._in_use + need + self._pool.cached_bytes() > self.budget:
            self._pool.drop_all()  # cached statevectors go back to the device first
        return True

    def _worker(self) -> None:
        stream = Stream()
        urgent = Stream(priority=-1000) if self.heavy_priority else stream
        while True:
            with self._work_cv:
                while not self._work and not self._stop:
                    self._work_cv.wait(timeout=0.1)
                if self._stop and not self._work:
                    return
                req, fut, t_arr, need, t_adm = self._work.popleft()
            try:
                z = self._execute(req, urgent if self._heavy(req) else stream)
                res = Result(req.rid, z, t_arr, t_adm, self.now(), req.circuit.n_qubits(),
                             req.precision, req.n_traj)
                fut.set_result(res)
            except Exception as e:  # the request fails, the engine keeps serving
                fut.set_exception(e)
            finally:
                with self._cv:
                    self._in_use -= need
                    self._active -= 1
                    self._cv.notify_all()

    def _batch_loop(self) -> None:
        """Runs every small request admitted since the last batch in one launch
        of the circuit-batch kernel, then completes them together."""
        stream = Stream()
        batch = CircuitBatch()
        while True:
            with self._bcv:
                while not self._bwork and not self._stop:
                    self._bcv.wait(timeout=0.1)
                if self._stop and not self._bwork:
                    return
                items = [self._bwork.popleft() for _ in range(min(len(self._bwork), self.max_batch))]
            if len(items) < self.batch_min:
                self._run_small_plain(items, stream)
                continue
            batch.clear()
            svs = []
            try:
                for req, *_ in items:
                    n = req.circuit.n_qubits()
                    fused = optimize_native(n, req.circuit.gates(),
                                            FusionConfig.size_only(self.batch_fusion_k))
                    sv = self._pool.get(n, req.precision)
                    svs.append(sv)
                    batch.add(sv, fused, init_zero=True)
                zs = batch.run(stream)
                done = self.now()
                for (req, fut, t_arr, _, t_adm), z in zip(items, zs):
                    fut.set_result(Result(req.rid, z, t_arr, t_adm, done, req.circuit.n_qubits(),
                                          req.precision, 0))
                self.batches_run += 1
                self.batched_requests += len(items)
            except Exception as e:  # the batch fails, the engine keeps serving
                try:
                    stream.sync()
                except Exception:
                    pass
                for _, fut, *_ in items:
                    if not fut.done():
                        fut.set_exception(e)
            finally:
                for sv in svs:
                    self._pool.put(sv)
                with self._cv:
                    for *_, need, _ in items:
                        self._in_use -= need
                    self._batched_active -= len(items)
                    self._cv.notify_all()

    def _run_small_plain(self, items, stream: Stream) -> None:
        """A batch below batch_min: its requests run one after another on the
        plain kernels, on the batcher's stream."""
        for req, fut, t_arr, need, t_adm in items:
            try:
                z = self._execute(req, stream)
                fut.set_result(Result(req.rid, z, t_arr, t_adm, self.now(), req.circuit.n_qubits(),
                                      req.precision, 0))
                self.small_plain_requests += 1
            except Exception as e:  # the request fails, the engine keeps serving
                fut.set_exception(e)
            finally:
                with self._cv:
                    self._in_use -= need
                    self._batched_active -= 1
                    self._cv.notify_all()

    def _execute(self, req: Request, stream: Stream) -> np.ndarray:
        """Host preparation, then the device phase (behind the heavy-request
        semaphore for requests that fill the GPU)."""
        prep = self._prepare(req)
        if self._heavy(req):
            with self._gpu_heavy:
                return self._launch(req, prep, stream)
        return self._launch(req, prep, stream)

    def _prepare(self, req: Request):
        """Fusion and program construction on the host: a trajectory program
        for a noisy request, a gate program for a pure one."""
        n = req.circuit.n_qubits()
        if req.n_traj:
            return TrajectoryProgram(req.circuit, self.traj_fusion_k or (3 if n <= 16 else 4))
        split = (req.precision == CudaPrecision.F32 and self.split_min_qubits > 0
                 and n >= self.split_min_qubits)
        fused = optimize_native(n, req.circuit.gates(),
                                FusionConfig.size_only(6 if split else self.fusion_k))
        tol = 1e-12 if req.precision == CudaPrecision.F64 else 1e-6
        prog = GateProgram(req.precision, n, tol, tol, split)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_program_add_fused(prog.handle, fused.handle, eb, L.ERR_LEN), eb,
                "program_add_fused")
        return prog

    def _launch(self, req: Request, prog, stream: Stream) -> np.ndarray:
        """Runs a prepared request on `stream` and returns its <Z_q>."""
        n = req.circuit.n_qubits()
        if req.n_traj:
            z, _ = prog.run(req.n_traj, req.seed, stream, True)
            return z.mean(axis=0)
        sv = self._pool.get(n, req.precision)
        ok = False
        try:
            sv.zero(stream)
            prog.run(sv, stream, self.use_graph)
            p1, nrm = qubit_populations(sv, stream)
            ok = True
            return (nrm - 2.0 * p1) / nrm
        finally:
            if not ok:
                # work of a failed request may still be queued on this stream:
                # let it drain before another worker can take the statevector
                try:
                    stream.sync()
                except Exception:
                    pass
            self._pool.put(sv)


# ── workload generation and the sequential plain-path baseline ──────────────


def make_stream(n_requests: int, rate_hz: float, seed: int, n_range=(10, 28), depth_range=(5, 40),
                noisy_frac: float = 0.2, n_traj: int = 256, noisy_max_qubits: int = 16,
                depolarizing: float = 1e-3) -> list[Request]:
    """Poisson arrivals of random brickwork circuits: qubits and depth uniform in
    the given ranges, half complex64 / half complex128, a fraction noisy
    (depolarizing p after every gate, n_traj trajectories, at most
    noisy_max_qubits qubits)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate_hz)
        noisy = rng.random() < noisy_frac
        n = int(rng.integers(n_range[0], (noisy_max_qubits if noisy else n_range[1]) + 1))
        d = int(rng.integers(depth_range[0], depth_range[1] + 1))
        prec = CudaPrecision.F32 if (noisy or rng.random() < 0.5) else CudaPrecision.F64
        circ = QuantumCircuit.brickwork(n, d, int(rng.integers(1 << 31)),
                                        depolarizing=depolarizing if noisy else 0.0)
        out.append(Request(circ, prec, n_traj if noisy else 0, int(rng.integers(1 << 31)), t, i))
    return out


def plain_service_time(req: Request) -> float:
    """Run one request alone on the plain per-gate path through the drop-in C ABI
    (compile_gate_ptx -> cubin_load -> kernel_launch for every unfused gate, the
    reference's execution of an unfused circuit; noisy requests run host-driven
    trajectories one by one) and return its wall time."""
    from .cuda import CudaKernelGenSpec, CudaKernelManager
    from .trajectory import run_plain

    t0 = time.perf_counter()
    n = req.circuit.n_qubits()
    if req.n_traj:
        run_plain(req.circuit, req.n_traj, req.seed)
        return time.perf_counter() - t0
    spec = CudaKernelGenSpec.f64() if req.precision == CudaPrecision.F64 else CudaKernelGenSpec.f32()
    mgr = CudaKernelManager(spec, timing=False)
    sv = CudaStatevector(n, req.precision)
    sv.zero()
    for g in req.circuit.gates():
        mgr.apply(mgr.generate(g), sv)
    mgr.sync()
    qubit_populations(sv)
    return time.perf_counter() - t0


def sequential_latencies(arrivals, service_times) -> np.ndarray:
    """Latencies of a single FIFO server that runs one request at a time."""
    free_at = 0.0
    out = []
    for a, s in zip(arrivals, service_times):
        start = max(a, free_at)
        free_at = start + s
        out.append(free_at - a)
    return np.array(out)


def latency_summary(lat) -> dict:
    lat = np.asarray(lat)
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "n": int(lat.size)}
