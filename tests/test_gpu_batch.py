"""Many small circuits in one persistent launch (cast_b200_batch_*): every
circuit of a mixed batch (qubit counts, depths, precisions, starting states)
against the oracle, the same result alone and in the batch, and <Z_q> against
the oracle's.  The reference runs such circuits one at a time
(src/simulator/mod.rs:523-547); its parity tolerances are 1e-10 (FP64) and 1e-5
(FP32) per amplitude (tests/cpu_cuda_compare.rs:27, 397)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cblib):
    from cast_simulator_b200 import cuda, fusion, simulator, types

    return cuda, fusion, simulator, types


def _z(psi):
    p = np.abs(psi) ** 2
    idx = np.arange(p.size)
    n = int(np.log2(p.size))
    return np.array([(p.sum() - 2 * p[(idx >> q) & 1 == 1].sum()) / p.sum() for q in range(n)])


def _cases(T, F):
    """(n, precision, fused gates, initial state or None) for a mixed batch."""
    out = []
    rng = np.random.default_rng(11)
    for i, n in enumerate([4, 7, 10, 12, 13, 16, 9, 14, 5, 11, 16, 8]):
        depth = int(rng.integers(3, 12))
        circ = T.QuantumCircuit.brickwork(n, depth, 100 + i)
        k = [2, 3, 4][i % 3]
        fused = F.optimize_native(n, circ.gates(), F.FusionConfig.size_only(k))
        prec = 1 if i % 2 == 0 else 0
        out.append((n, prec, circ, fused, i % 3 == 2))
    return out


def test_mixed_batch_matches_oracle_and_runs_alone(mods, oracle):
    cu, F, S, T = mods
    cases = _cases(T, F)
    batch = S.CircuitBatch()
    svs, refs, inits = [], [], []
    for j, (n, prec, circ, fused, from_state) in enumerate(cases):
        sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
        init = oracle.random_state(n, 500 + j) if from_state else None
        if init is not None:
            sv.upload(init)
        batch.add(sv, fused, init_zero=init is None)
        svs.append(sv)
        inits.append(init)
        refs.append(oracle.simulate(n, [(g.matrix(), g.qubits()) for g in circ.gates()], init))
    zs = batch.run()
    assert len(zs) == len(cases)
    got = [sv.download() for sv in svs]
    for (n, prec, *_), psi, ref, z in zip(cases, got, refs, zs):
        tol = 1e-10 if prec == 1 else 1e-5
        assert np.max(np.abs(psi - ref)) < tol, (n, prec)
        assert np.max(np.abs(z - _z(ref))) < (1e-10 if prec == 1 else 1e-5)
    # each circuit alone (a batch of one) gives the same bits as in the mix
    for (n, prec, circ, fused, _), init, psi_mix, z_mix in zip(cases, inits, got, zs):
        one = S.CircuitBatch()
        sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
        if init is not None:
            sv.upload(init)
        one.add(sv, fused, init_zero=init is None)
        z1 = one.run()[0]
        assert np.array_equal(sv.download(), psi_mix)
        assert np.array_equal(z1, z_mix)


def test_batch_reuse_and_gate_lists(mods, oracle):
    """A batch object runs, clears and runs again (its device buffers are reused
    and grown); plain gate lists with unfused gates work too."""
    cu, F, S, T = mods
    batch = S.CircuitBatch()
    for rounds in range(3):
        batch.clear()
        svs, refs = [], []
        for j in range(5 + 20 * rounds):
            n = 6 + (j % 8)
            circ = T.QuantumCircuit.brickwork(n, 4 + (j % 3), 7 * j + rounds)
            sv = cu.CudaStatevector(n, cu.CudaPrecision.F64)
            batch.add(sv, circ.gates())
            svs.append(sv)
            refs.append(oracle.simulate(n, [(g.matrix(), g.qubits()) for g in circ.gates()]))
        zs = batch.run()
        for sv, ref, z in zip(svs, refs, zs):
            assert np.max(np.abs(sv.download() - ref)) < 1e-10
            assert np.max(np.abs(z - _z(ref))) < 1e-10


def test_batch_rejects_bad_circuits(mods):
    from cast_simulator_b200 import _lib as L

    cu, F, S, T = mods
    batch = S.CircuitBatch()
    sv = cu.CudaStatevector(8, cu.CudaPrecision.F64)
    wide = T.QuantumCircuit.brickwork(8, 4, 1)
    fused5 = F.optimize_native(8, wide.gates(), F.FusionConfig.size_only(5))
    if any(len(g.qubits()) > 4 for g in fused5.gates()):
        with pytest.raises(L.CudaError, match="wider"):
            batch.add(sv, fused5)
    big = cu.CudaStatevector(21, cu.CudaPrecision.F32)
    with pytest.raises(L.CudaError, match="qubits"):
        batch.add(big, [])

    class G:
        def __init__(self, m, q):
            self._m, self._q = m, q

        def matrix(self):
            return self._m

        def qubits(self):
            return self._q

    with pytest.raises(L.CudaError, match="ascending"):
        batch.add(sv, [G(np.eye(4), (3, 1))])
    with pytest.raises(L.CudaError, match="below"):
        batch.add(sv, [G(np.eye(2), (8,))])
    batch.clear()
    batch.add(sv, [G(np.eye(2), (0,))])
    batch.add(sv, [G(np.eye(2), (1,))])  # the same statevector twice
    with pytest.raises(L.CudaError, match="share"):
        batch.run()
