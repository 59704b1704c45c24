"""Host-side logic of the serving loop, without a GPU: the arrival stream the
bench draws, the admission charge of a request, and the single-server FIFO
model the sequential plain-path baseline uses, and the scheduler (admission by
memory and slots in arrival order, failure isolation, shutdown) with the
device work replaced by a host fake."""
import numpy as np
import pytest

from cast_simulator_b200 import serving as S
from cast_simulator_b200.cuda import CudaPrecision
from cast_simulator_b200.types import QuantumCircuit


def test_stream_shape():
    reqs = S.make_stream(400, 40.0, 7, n_range=(10, 24))
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    # Poisson arrivals: mean gap 1 / rate
    assert abs(np.diff(np.concatenate([[0.0], arr])).mean() - 1 / 40.0) < 0.2 / 40.0
    noisy = [r for r in reqs if r.n_traj]
    assert 0.1 < len(noisy) / len(reqs) < 0.3 and all(r.n_traj == 256 for r in noisy)
    assert all(10 <= r.circuit.n_qubits() <= 16 for r in noisy)
    assert all(r.precision == CudaPrecision.F32 for r in noisy)
    clean = [r for r in reqs if not r.n_traj]
    assert all(10 <= r.circuit.n_qubits() <= 24 for r in clean)
    f64 = sum(r.precision == CudaPrecision.F64 for r in clean) / len(clean)
    assert 0.35 < f64 < 0.65
    # same seed, same stream
    again = S.make_stream(400, 40.0, 7, n_range=(10, 24))
    assert [(r.arrival, r.circuit.n_qubits(), r.n_traj) for r in again] == \
        [(r.arrival, r.circuit.n_qubits(), r.n_traj) for r in reqs]


def test_request_bytes_charge():
    c20 = QuantumCircuit.brickwork(20, 2, 1)
    assert S.request_bytes(S.Request(c20, CudaPrecision.F64)) == 16 << 20
    assert S.request_bytes(S.Request(c20, CudaPrecision.F32)) == 8 << 20
    c12 = QuantumCircuit.brickwork(12, 2, 1, depolarizing=1e-3)
    # trajectories: one complex64 slice per CTA in flight plus the <Z> rows
    r = S.Request(c12, CudaPrecision.F32, n_traj=256)
    assert S.request_bytes(r, sm_count=148) == (8 << 12) * 148 + 8 * 256 * 13
    assert S.request_bytes(S.Request(c12, CudaPrecision.F32, n_traj=64), sm_count=148) == \
        (8 << 12) * 64 + 8 * 64 * 13


def test_sequential_fifo_model():
    # idle server: latency = service time; busy server: requests queue
    lat = S.sequential_latencies([0.0, 10.0, 10.5, 11.0], [1.0, 2.0, 2.0, 0.5])
    assert lat.tolist() == pytest.approx([1.0, 2.0, 3.5, 3.5])
    summ = S.latency_summary([0.010, 0.020, 0.030, 0.040])
    assert summ["n"] == 4 and summ["p50_ms"] == pytest.approx(25.0)
    assert summ["mean_ms"] == pytest.approx(25.0) and summ["p99_ms"] <= 40.0


# ── the scheduler, with the device work replaced by a fake ──────────────────


class _FakeStream:
    def sync(self):
        pass


@pytest.fixture
def fake_engine(monkeypatch):
    """A ServingEngine whose per-request work is a short sleep on the host: it
    records the order requests start in and the largest number running at once,
    and raises for requests whose seed is negative."""
    import threading
    import time

    state = {"running": 0, "peak": 0, "order": [], "lock": threading.Lock()}

    def execute(self, req, stream):
        with state["lock"]:
            state["running"] += 1
            state["peak"] = max(state["peak"], state["running"])
            state["order"].append(req.rid)
        try:
            time.sleep(0.02)
            if req.seed < 0:
                raise RuntimeError(f"request {req.rid} failed")
            return np.full(req.circuit.n_qubits(), float(req.rid))
        finally:
            with state["lock"]:
                state["running"] -= 1

    monkeypatch.setattr(S, "Stream", _FakeStream)
    monkeypatch.setattr(S.ServingEngine, "_execute", execute)
    engines = []

    def make(**kw):
        kw.setdefault("batch_max_qubits", 0)  # every request on the worker path
        eng = S.ServingEngine(**kw)
        engines.append(eng)
        return eng

    yield make, state
    for eng in engines:
        eng.shutdown()


def _reqs(n_qubits, count, prec=CudaPrecision.F64, seeds=None):
    c = QuantumCircuit.brickwork(n_qubits, 2, 1)
    return [S.Request(c, prec, 0, (seeds or {}).get(i, i), 0.0, i) for i in range(count)]


def test_admission_is_bounded_by_the_memory_budget(fake_engine):
    make, state = fake_engine
    one = 16 << 20  # a 20-qubit complex128 statevector
    eng = make(max_slots=8, mem_budget_bytes=int(2.5 * one))
    res = [f.result(timeout=30) for f in [eng.submit(r) for r in _reqs(20, 8)]]
    assert [r.rid for r in res] == list(range(8))
    assert all(np.all(r.z == r.rid) for r in res)
    assert state["peak"] <= 2 and eng.max_concurrent <= 2
    assert all(r.admitted >= r.arrival and r.finished >= r.admitted for r in res)
    assert eng._in_use == 0 and eng._active == 0


def test_admission_is_bounded_by_slots_and_keeps_arrival_order(fake_engine):
    make, state = fake_engine
    eng = make(max_slots=3, mem_budget_bytes=1 << 40)
    futs = [eng.submit(r) for r in _reqs(12, 12)]
    for f in futs:
        f.result(timeout=30)
    assert state["peak"] <= 3 and eng.max_concurrent == 3
    # admission never reorders: with one slot, requests start in submission order
    make2, state2 = fake_engine
    state["order"].clear()
    eng1 = make2(max_slots=1, mem_budget_bytes=1 << 40)
    for f in [eng1.submit(r) for r in _reqs(10, 6)]:
        f.result(timeout=30)
    assert state["order"] == list(range(6))


def test_a_failing_request_does_not_stop_the_engine(fake_engine):
    make, state = fake_engine
    eng = make(max_slots=2, mem_budget_bytes=1 << 40)
    futs = [eng.submit(r) for r in _reqs(10, 6, seeds={2: -1})]
    for i, f in enumerate(futs):
        if i == 2:
            with pytest.raises(RuntimeError, match="request 2 failed"):
                f.result(timeout=30)
        else:
            assert f.result(timeout=30).rid == i
    assert eng._in_use == 0 and eng._active == 0


def test_oversized_requests_and_shutdown(fake_engine):
    make, state = fake_engine
    eng = make(max_slots=1, mem_budget_bytes=(16 << 20) + 1)
    with pytest.raises(ValueError, match="budget"):
        eng.submit(_reqs(21, 1)[0])
    futs = [eng.submit(r) for r in _reqs(20, 5)]
    futs[0].result(timeout=30)
    eng.shutdown()
    done = failed = 0
    for f in futs:
        try:
            f.result(timeout=30)
            done += 1
        except RuntimeError as e:
            assert "shut down" in str(e)
            failed += 1
    # admitted requests finish, the rest fail instead of waiting for ever
    assert done >= 1 and done + failed == 5
    with pytest.raises(RuntimeError, match="shut down"):
        eng.submit(_reqs(20, 1)[0])


class _FakeSv:
    def __init__(self, n, prec):
        self.n, self.prec = n, prec

    def n_qubits(self):
        return self.n

    def precision(self):
        return self.prec

    def nbytes(self):
        return (16 if self.prec == CudaPrecision.F64 else 8) << self.n


def test_small_batches_run_on_the_plain_path(fake_engine, monkeypatch):
    """Below batch_min the batcher runs its requests one after another on the
    plain path (never the batch kernel); a failing request fails alone and the
    memory returns to the budget."""

    class NoBatch:
        def clear(self):
            raise AssertionError("the batch kernel must not run for small batches")

        run = add = clear

    make, state = fake_engine
    monkeypatch.setattr(S, "CircuitBatch", NoBatch)
    eng = make(max_slots=2, mem_budget_bytes=1 << 40, batch_max_qubits=12, batch_min=1 << 20)
    futs = [eng.submit(r) for r in _reqs(10, 12, seeds={4: -1})]
    for i, f in enumerate(futs):
        if i == 4:
            with pytest.raises(RuntimeError, match="request 4 failed"):
                f.result(timeout=30)
        else:
            r = f.result(timeout=30)
            assert r.rid == i and np.all(r.z == float(i))
    assert eng.small_plain_requests == 11 and eng.batches_run == 0
    assert state["peak"] == 1  # one after another on the batcher thread
    assert eng._in_use == 0 and eng._batched_active == 0


def test_small_requests_run_batched(monkeypatch):
    """Small pure requests go to the batcher, which runs every request admitted
    while its previous launch ran in one batch; a failing batch fails only its
    own requests; memory returns to the budget."""
    import threading
    import time

    runs = []

    class FakeBatch:
        def __init__(self):
            self.items = []

        def clear(self):
            self.items = []

        def add(self, sv, fused, init_zero=True):
            self.items.append(sv)

        def run(self, stream=None):
            time.sleep(0.05)
            runs.append(len(self.items))
            if any(getattr(sv, "poison", False) for sv in self.items):
                raise RuntimeError("batch failed")
            return [np.full(sv.n, float(len(runs))) for sv in self.items]

    pool_lock = threading.Lock()

    def pool_get(self, n, prec):
        with pool_lock:
            return _FakeSv(n, prec)

    monkeypatch.setattr(S, "Stream", _FakeStream)
    monkeypatch.setattr(S, "CircuitBatch", FakeBatch)
    monkeypatch.setattr(S._SvPool, "get", pool_get)
    eng = S.ServingEngine(max_slots=2, mem_budget_bytes=1 << 40, batch_max_qubits=12, batch_min=1)
    try:
        futs = [eng.submit(r) for r in _reqs(10, 40)]
        res = [f.result(timeout=30) for f in futs]
        assert [r.rid for r in res] == list(range(40))
        assert sum(runs) == 40 and len(runs) < 40  # requests were grouped
        assert eng.batched_requests == 40 and eng.batches_run == len(runs)
        assert eng._in_use == 0 and eng._batched_active == 0 and eng._active == 0
        # a failing batch fails its requests, later ones are served
        orig = pool_get

        def poisoned(self, n, prec):
            sv = orig(self, n, prec)
            sv.poison = True
            return sv

        monkeypatch.setattr(S._SvPool, "get", poisoned)
        bad = eng.submit(_reqs(10, 1)[0])
        with pytest.raises(RuntimeError, match="batch failed"):
            bad.result(timeout=30)
        monkeypatch.setattr(S._SvPool, "get", pool_get)
        assert eng.submit(_reqs(10, 1)[0]).result(timeout=30).rid == 0
        assert eng._in_use == 0 and eng._batched_active == 0
    finally:
        eng.shutdown()


def test_heavy_requests_run_one_at_a_time_on_the_device(monkeypatch):
    """Requests that fill the GPU (here pure requests of 14+ qubits) never run
    their device phase together when heavy_slots = 1, but they are admitted and
    prepared meanwhile, and small requests overlap with them."""
    import threading
    import time

    st = {"heavy": 0, "heavy_peak": 0, "all": 0, "all_peak": 0, "prepared_while_heavy": 0,
          "lock": threading.Lock()}

    def prepare(self, req):
        with st["lock"]:
            if st["heavy"]:
                st["prepared_while_heavy"] += 1
        return None

    def launch(self, req, prep, stream):
        heavy = req.circuit.n_qubits() >= 14
        with st["lock"]:
            st["all"] += 1
            st["all_peak"] = max(st["all_peak"], st["all"])
            if heavy:
                st["heavy"] += 1
                st["heavy_peak"] = max(st["heavy_peak"], st["heavy"])
        try:
            time.sleep(0.03)
            return np.zeros(req.circuit.n_qubits())
        finally:
            with st["lock"]:
                st["all"] -= 1
                if heavy:
                    st["heavy"] -= 1

    monkeypatch.setattr(S, "Stream", _FakeStream)
    monkeypatch.setattr(S.ServingEngine, "_prepare", prepare)
    monkeypatch.setattr(S.ServingEngine, "_launch", launch)
    eng = S.ServingEngine(max_slots=6, mem_budget_bytes=1 << 50, batch_max_qubits=0, heavy_slots=1,
                          heavy_pure_qubits=14)
    try:
        reqs = [S.Request(QuantumCircuit.brickwork(15 if i % 2 == 0 else 10, 2, 1), CudaPrecision.F64,
                          0, i, 0.0, i) for i in range(12)]
        for f in [eng.submit(r) for r in reqs]:
            f.result(timeout=30)
        assert st["heavy_peak"] == 1  # heavy device phases never overlapped
        assert st["all_peak"] >= 2  # small requests ran beside a heavy one
        assert st["prepared_while_heavy"] >= 1  # requests were prepared meanwhile
        assert eng._active == 0 and eng._in_use == 0
    finally:
        eng.shutdown()
