"""Continuous-batching serving loop: every result is the same alone and in the
mix (FP64 1e-12, FP32 1e-6; trajectories are seeded and bit-identical), memory
admission holds, failures stay local to their request."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cblib):
    from cast_simulator_b200 import cuda, serving, types

    return cuda, serving, types


def _mix(S, T, cu):
    rng = np.random.default_rng(12)
    reqs = []
    for i in range(24):
        n = int(rng.integers(8, 15))
        noisy = i % 6 == 5
        prec = cu.CudaPrecision.F32 if (noisy or i % 2) else cu.CudaPrecision.F64
        circ = T.QuantumCircuit.brickwork(n, int(rng.integers(3, 12)), int(rng.integers(1 << 30)),
                                          depolarizing=0.01 if noisy else 0.0)
        reqs.append(S.Request(circ, prec, 64 if noisy else 0, 1000 + i, 0.0, i))
    return reqs


def test_results_same_alone_and_in_mix(mods, oracle):
    """The mix runs with small requests batched into the circuit-batch kernel
    and the others on worker streams.  Each result equals (bit for bit) the
    same request submitted alone to the same kind of engine, and (within
    tolerance) the request run alone on the worker path with batching off."""
    cu, S, T = mods
    reqs = _mix(S, T, cu)
    eng = S.ServingEngine(max_slots=6, batch_min=1)
    try:
        mixed = eng.run_stream(reqs)
        assert eng.max_concurrent > 1
        assert eng.batched_requests == sum(1 for r in reqs if not r.n_traj)
        assert eng.batches_run < eng.batched_requests  # grouped into fewer launches
    finally:
        eng.shutdown()
    solo_eng = S.ServingEngine(max_slots=1, batch_min=1)
    try:
        alone = [solo_eng.submit(r).result() for r in reqs]
    finally:
        solo_eng.shutdown()
    plain_eng = S.ServingEngine(max_slots=1, batch_max_qubits=0)
    try:
        plain = [plain_eng.submit(r).result() for r in reqs]
    finally:
        plain_eng.shutdown()
    for m, a, pl, r in zip(mixed, alone, plain, reqs):
        assert m.rid == a.rid == pl.rid == r.rid
        assert np.array_equal(m.z, a.z)
        tol = 1e-12 if r.precision == cu.CudaPrecision.F64 else 1e-5
        if r.n_traj:
            assert np.array_equal(m.z, pl.z)
        else:
            assert np.max(np.abs(m.z - pl.z)) < tol
    # pure requests against the CPU oracle
    for m, r in zip(mixed, reqs):
        if r.n_traj:
            continue
        n = r.circuit.n_qubits()
        sv = oracle.simulate(n, [(g.matrix(), g.qubits()) for g in r.circuit.gates()])
        p = np.abs(sv) ** 2
        idx = np.arange(p.size)
        z = np.array([1 - 2 * p[(idx >> q) & 1 == 1].sum() for q in range(n)])
        assert np.max(np.abs(m.z - z)) < (1e-10 if r.precision == cu.CudaPrecision.F64 else 1e-5)


def test_memory_admission_limits_concurrency(mods):
    cu, S, T = mods
    n = 16
    reqs = [S.Request(T.QuantumCircuit.brickwork(n, 4, i), cu.CudaPrecision.F64, 0, i, 0.0, i)
            for i in range(8)]
    one = S.request_bytes(reqs[0])
    eng = S.ServingEngine(max_slots=8, mem_budget_bytes=2 * one)
    try:
        res = eng.run_stream(reqs)
        assert len(res) == 8 and eng.max_concurrent <= 2
        with pytest.raises(ValueError, match="budget"):
            eng.submit(S.Request(T.QuantumCircuit.brickwork(18, 2, 1), cu.CudaPrecision.F64))
    finally:
        eng.shutdown()


def test_failed_request_does_not_stop_the_engine(mods):
    cu, S, T = mods
    eng = S.ServingEngine(max_slots=2)
    try:
        bad = S.Request(T.QuantumCircuit.brickwork(23, 2, 1, depolarizing=0.01), cu.CudaPrecision.F32,
                        8, 1, 0.0, 0)  # trajectories support at most 22 qubits
        good = S.Request(T.QuantumCircuit.brickwork(10, 3, 2), cu.CudaPrecision.F64, 0, 2, 0.0, 1)
        fb, fg = eng.submit(bad), eng.submit(good)
        with pytest.raises(Exception, match="1..22"):
            fb.result()
        assert fg.result().z.shape == (10,)
    finally:
        eng.shutdown()


def test_large_complex64_requests_use_the_tensor_path(mods, oracle):
    """A complex64 request of split_min_qubits or more runs as a split-precision
    program (k = 6 on the tensor cores); its <Z_q> stays within the tensor
    path's error of the oracle, and with the split turned off the engine gives
    the plain path's result."""
    cu, S, T = mods
    n = 20
    circ = T.QuantumCircuit.brickwork(n, 6, 77)
    req = S.Request(circ, cu.CudaPrecision.F32, 0, 1, 0.0, 0)
    sv = oracle.simulate(n, [(g.matrix(), g.qubits()) for g in circ.gates()])
    p = np.abs(sv) ** 2
    idx = np.arange(p.size)
    z_ref = np.array([1 - 2 * p[(idx >> q) & 1 == 1].sum() for q in range(n)])
    for split_min, tol in ((20, 1e-4), (0, 1e-5)):
        eng = S.ServingEngine(max_slots=2, split_min_qubits=split_min)
        try:
            z = eng.submit(req).result().z
        finally:
            eng.shutdown()
        assert np.max(np.abs(z - z_ref)) < tol, (split_min, np.max(np.abs(z - z_ref)))
