"""Host-side logic of the serving loop, without a GPU: the arrival stream the
bench draws, the admission charge of a request, and the single-server FIFO
model the sequential plain-path baseline uses."""
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
