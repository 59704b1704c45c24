"""GPU parity of the gate path through the drop-in C ABI vs the CPU oracle.

Tolerances are the reference's (tests/cpu_cuda_compare.rs:27, 397): 1e-10 per
amplitude for FP64, 1e-5 for FP32; 1e-9 for sequential circuits
(tests/circuit_execution_order.rs:34)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = {1: 1e-10, 0: 1e-5}


@pytest.fixture(scope="module")
def cu(cblib):
    from cast_simulator_b200 import cuda

    return cuda


def run_gates(cu, n, gates, init, prec):
    spec = cu.CudaKernelGenSpec.f64() if prec == 1 else cu.CudaKernelGenSpec.f32()
    mgr = cu.CudaKernelManager(spec)
    sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
    sv.upload(init)
    for g in gates:
        mgr.apply(mgr.generate(g), sv)
    mgr.sync()
    return sv.download()


class _G:
    def __init__(self, m, q):
        self._m, self._q = np.ascontiguousarray(m), tuple(q)

    def matrix(self):
        return self._m

    def qubits(self):
        return self._q


def haar(rng, d):
    z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


@pytest.mark.parametrize("prec", [1, 0])
@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6, 7])
def test_single_gate_all_placements(cu, oracle, prec, k):
    rng = np.random.default_rng(100 + k)
    for n in sorted({k, min(k + 2, 20), 12, 17}):
        if n < k:
            continue
        placements = [tuple(range(k)), tuple(range(n - k, n))]
        for _ in range(3):
            placements.append(tuple(sorted(rng.choice(n, size=k, replace=False).tolist())))
        for q in placements:
            m = haar(rng, 1 << k)
            init = oracle.random_state(n, 5 + k)
            ref = init.copy()
            oracle.apply_gate(ref, m, q)
            got = run_gates(cu, n, [_G(m, q)], init, prec)
            err = np.max(np.abs(got - ref))
            assert err < TOL[prec], (n, q, err)


@pytest.mark.parametrize("prec", [1, 0])
def test_random_circuit_sequence(cu, oracle, prec):
    """Random 1q/2q/3q Haar circuits, 14 qubits, 80 gates (circuit_execution_order.rs)."""
    rng = np.random.default_rng(7)
    n = 14
    gates = []
    for _ in range(80):
        k = int(rng.integers(1, 4))
        q = tuple(sorted(rng.choice(n, size=k, replace=False).tolist()))
        gates.append((haar(rng, 1 << k), q))
    init = oracle.random_state(n, 3)
    ref = oracle.simulate(n, gates, init)
    got = run_gates(cu, n, [_G(m, q) for m, q in gates], init, prec)
    assert np.max(np.abs(got - ref)) < (1e-9 if prec == 1 else 1e-4)
    rep = oracle.fidelity_report(ref, got)
    assert rep["one_minus_abs_overlap"] < (1e-12 if prec == 1 else 1e-5)


def test_qft14_golden_on_gpu(cu, oracle):
    golden = np.load(os.path.join(GOLDEN, "qft14_seeded.npy"))
    got = run_gates(cu, 14, [_G(m, q) for m, q in oracle.qft_cx(14)], oracle.seeded_state(14), 1)
    assert np.max(np.abs(got - golden)) < 1e-10


def _monomial(rng, k):
    """A permutation with unit phases: one nonzero a row (fused CX / phase blocks)."""
    d = 1 << k
    m = np.zeros((d, d), dtype=complex)
    m[np.arange(d), rng.permutation(d)] = np.exp(2j * np.pi * rng.random(d))
    return m


def _block_sparse(rng, k):
    """Identity on k - 2 qubits times a dense 2-qubit gate: 4 nonzeros a row."""
    return np.kron(np.eye(1 << (k - 2)), haar(rng, 4))


@pytest.mark.parametrize("prec", [1, 0])
@pytest.mark.parametrize("k", [3, 4, 5, 6, 7])
def test_sparse_gates_all_placements(cu, oracle, prec, k):
    """Gates with at most 2^k / 4 nonzeros a row (CSR kernel from k = 5, dense
    kernels below): monomial and block-sparse matrices, low, high and random
    targets, small and partial grids (fewer groups than a CTA holds)."""
    rng = np.random.default_rng(300 + k)
    for n in sorted({k, k + 1, 12, 17}):
        placements = [tuple(range(k)), tuple(range(n - k, n))]
        placements.append(tuple(sorted(rng.choice(n, size=k, replace=False).tolist())))
        for q in placements:
            for make in (_monomial, _block_sparse):
                m = make(rng, k)
                init = oracle.random_state(n, 11 + k)
                ref = init.copy()
                oracle.apply_gate(ref, m, q)
                got = run_gates(cu, n, [_G(m, q)], init, prec)
                err = np.max(np.abs(got - ref))
                assert err < TOL[prec], (n, q, make.__name__, err)


@pytest.mark.parametrize("prec", [1, 0])
def test_sparse_gates_with_empty_rows(cu, oracle, prec):
    """Non-unitary sparse matrices (a projector on one wire of a 5-qubit block,
    and the zero matrix): rows without nonzeros write exact zeros, in both the
    direct (high targets) and the tiled (low targets) CSR kernels."""
    rng = np.random.default_rng(17)
    proj = np.kron(np.eye(16), np.diag([1.0, 0.0])).astype(complex)  # rows of |1> on wire 0 empty
    zero = np.zeros((32, 32), dtype=complex)
    n = 13
    for m in (proj, zero):
        for q in ((0, 1, 2, 3, 4), (8, 9, 10, 11, 12)):
            init = oracle.random_state(n, int(rng.integers(100)))
            ref = init.copy()
            oracle.apply_gate(ref, m, q)
            got = run_gates(cu, n, [_G(m, q)], init, prec)
            assert np.max(np.abs(got - ref)) < TOL[prec], q
            assert np.all(got[ref == 0] == 0)


def test_sparse_gates_in_programs(cu, oracle):
    """The gate-program path (graph replay, split precision on) routes sparse
    5- and 6-qubit gates to the CSR kernel in exact FP32."""
    from cast_simulator_b200.simulator import GateProgram, Stream

    rng = np.random.default_rng(5)
    n = 16
    gates = [(_monomial(rng, 6), (0, 3, 5, 9, 12, 15)), (_block_sparse(rng, 5), (1, 2, 7, 8, 14)),
             (haar(rng, 8), (4, 6, 10))]
    init = oracle.random_state(n, 2)
    ref = oracle.simulate(n, gates, init)
    for split in (False, True):
        prog = GateProgram(cu.CudaPrecision.F32, n, 1e-6, 1e-6, split)
        for m, q in gates:
            prog.add(m, q)
        sv = cu.CudaStatevector(n, cu.CudaPrecision.F32)
        sv.upload(init)
        st = Stream()
        prog.run(sv, st, use_graph=True)
        st.sync()
        assert np.max(np.abs(sv.download() - ref)) < 1e-5


def test_sparse_entries_snapped(cu, oracle):
    """Scalars within ztol/K of 0 and otol/K of +-1 behave as exact 0 / +-1
    (cuda_gen.cpp:84-103): the GPU matches the oracle run on the snapped matrix."""
    m = np.array([[1 + 1e-14, 2e-14j], [3e-14, -1 - 1e-14j]], dtype=complex)
    init = oracle.random_state(10, 1)
    ref = init.copy()
    oracle.apply_gate(ref, oracle.snap(m, 1e-12, 1e-12), [4])
    got = run_gates(cu, 10, [_G(m, [4])], init, 1)
    assert np.max(np.abs(got - ref)) < 1e-15


@pytest.mark.parametrize("prec", [1, 0])
def test_statevector_memory_and_reductions(cu, oracle, prec):
    n = 15
    sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
    sv.zero()
    z = sv.download()
    assert z[0] == 1 and np.count_nonzero(z) == 1
    init = oracle.random_state(n, 9) * 3.0
    sv.upload(init)
    back = sv.download()
    assert np.max(np.abs(back - init)) < (1e-15 if prec else 1e-6)
    assert abs(sv.norm_squared() - 9.0) < (1e-12 if prec else 1e-5)
    sv.normalize()
    assert abs(sv.norm_squared() - 1.0) < (1e-12 if prec else 1e-5)
    c = sv.clone_device()
    assert np.array_equal(c.download(), sv.download())


def test_tiny_statevectors(cu, oracle):
    """n = k edge cases and the scalar tail of the reductions (n = 0, 1)."""
    for n in (1, 2):
        sv = cu.CudaStatevector(n, cu.CudaPrecision.F32)
        sv.upload(oracle.random_state(n, 2))
        assert abs(sv.norm_squared() - 1) < 1e-6


def test_launch_errors(cu):
    mgr = cu.CudaKernelManager(cu.CudaKernelGenSpec.f64())
    kid = mgr.generate(_G(np.eye(4), (2, 5)))
    sv = cu.CudaStatevector(4, cu.CudaPrecision.F64)
    with pytest.raises(ValueError, match="outside"):
        mgr.apply(kid, sv)
