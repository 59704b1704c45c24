"""Pin the CPU oracle to the reference: golden vectors derived from the
reference's own fixture (tests/assets/qft_14.qasm) and the reference's
known-answer tests, restated."""
import json
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_qft14_golden_matches_fixture_semantics(oracle):
    """Oracle QFT-CX builder + gate semantics == independent interpreter run of
    the reference's qft_14.qasm on the reference test input."""
    meta = json.load(open(os.path.join(GOLDEN, "qft14_meta.json")))
    golden = np.load(os.path.join(GOLDEN, "qft14_seeded.npy"))
    gates = oracle.qft_cx(14)
    assert len(gates) == sum(meta["gate_counts"].values()) == 476
    out = oracle.simulate(14, gates, oracle.seeded_state(14))
    assert np.max(np.abs(out - golden)) < 1e-12
    rep = oracle.fidelity_report(golden, out)
    assert rep["one_minus_abs_overlap"] < 1e-12


def test_qft_cx_equals_qft_cp(oracle):
    """Decomposed controlled phases reproduce QuantumCircuit::qft (circuit.rs:151-171)."""
    init = oracle.random_state(10, 7)
    a = oracle.simulate(10, oracle.qft_cx(10), init)
    b = oracle.simulate(10, oracle.qft_cp(10, True), init)
    assert np.max(np.abs(a - b)) < 1e-12


def test_h_and_x_on_zero(oracle):
    """src/cuda/tests.rs:109-165: H|0> = (|0>+|1>)/sqrt2, X|0> = |1>."""
    sv = oracle.zero_state(3)
    oracle.apply_gate(sv, oracle.named(oracle.H), [0])
    s = 1 / math.sqrt(2)
    assert np.allclose(sv[:2], [s, s], atol=1e-10) and np.allclose(sv[2:], 0)
    sv = oracle.zero_state(3)
    oracle.apply_gate(sv, oracle.named(oracle.X), [2])
    assert abs(sv[4] - 1) < 1e-10 and np.count_nonzero(np.abs(sv) > 1e-12) == 1


def test_h_squared_is_identity(oracle):
    """tests/cpu_cuda_compare.rs:280-315."""
    init = oracle.seeded_state(6)
    sv = init.copy()
    h = oracle.named(oracle.H)
    oracle.apply_gate(sv, h, [3])
    oracle.apply_gate(sv, h, [3])
    assert np.max(np.abs(sv - init)) < 1e-10


def test_qft_zero_state_uniform_and_swap_bit_reversal(oracle):
    """circuit.rs:201-271: QFT|0> uniform; the swaps bit-reverse amplitudes."""
    n = 8
    pops = np.abs(oracle.simulate(n, oracle.qft_cp(n, True))) ** 2
    assert np.max(np.abs(pops - 1 / 256)) < 1e-10
    one = oracle.zero_state(n)
    oracle.apply_gate(one, oracle.named(oracle.X), [0])
    a = oracle.simulate(n, oracle.qft_cp(n, True), one)
    b = oracle.simulate(n, oracle.qft_cp(n, False), one)
    rev = [int(format(j, f"0{n}b")[::-1], 2) for j in range(1 << n)]
    assert np.max(np.abs(a - b[rev])) < 1e-10


def test_pdep_worked_example(oracle):
    """The worked example of cuda_gen.cpp:156-170: targets {2,4,5}, combo 0b11001."""
    mask = ~((1 << 2) | (1 << 4) | (1 << 5)) & ((1 << 64) - 1)
    got = oracle.pdep(0b11001, mask)
    # bits 0,1 <- 0b01; bit 3 <- 0; bits 6,7 <- 0b11
    assert got == (0b01 | (0 << 3) | (0b11 << 6))


def test_canonicalize_example(oracle):
    """gate.rs:690-708: X(x)I given on qubits [1,0] equals I(x)X on [0,1]."""
    m = np.array([[0, 1, 0, 0], [1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex)
    got, q = oracle.canonicalize(m, [1, 0])
    exp = np.array([[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]], dtype=complex)
    assert q == (0, 1) and np.array_equal(got, exp)
    with pytest.raises(ValueError, match="distinct"):
        oracle.canonicalize(np.eye(4, dtype=complex), [0, 0])


def test_matmul_known_answers(oracle):
    """gate.rs:722-780: involution, disjoint, non-adjacent and overlapping products."""
    x = oracle.named(oracle.X)
    m, q = oracle.matmul((x, [0]), (x, [0]))
    assert q == (0,) and np.array_equal(m, np.eye(2))
    m, q = oracle.matmul((x, [1]), (x, [0]))
    assert q == (0, 1) and np.array_equal(m, np.fliplr(np.eye(4)))
    m, q = oracle.matmul((x, [0]), (x, [2]))
    assert q == (0, 2) and np.array_equal(m, np.fliplr(np.eye(4)))
    m, q = oracle.matmul((x, [1]), (np.eye(4, dtype=complex), [0, 1]))
    exp = np.array([[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]], dtype=complex)
    assert q == (0, 1) and np.array_equal(m, exp)


def test_fused_equals_sequential(oracle):
    """Fusion invariance (tests/fusion_correctness.rs:24, tol 1e-10)."""
    rng = np.random.default_rng(3)
    init = oracle.random_state(9, 11)
    gates = oracle.brickwork(9, 4, 5)
    seq = oracle.simulate(9, gates, init)
    fused = gates[0]
    for g in gates[1:4]:
        fused = oracle.matmul(g, fused)
    rest = gates[4:]
    out = oracle.simulate(9, [fused] + rest, init)
    assert np.max(np.abs(out - seq)) < 1e-10
    del rng


def test_depolarizing_density_matrix_known_answer(oracle):
    """tests/density_matrix.rs:85-113: rho00 = 1 - 2p/3 after depolarizing(p) on |0>."""
    p, n = 0.15, 2
    rho = oracle.dm_zero(n)
    kr = [oracle.named(oracle.I), oracle.named(oracle.X), oracle.named(oracle.Y), oracle.named(oracle.Z)]
    oracle.dm_apply_channel(rho, n, kr, [1 - p, p / 3, p / 3, p / 3], [0])
    diag = oracle.dm_populations(rho, n)
    assert abs(diag.sum() - 1) < 1e-10
    assert abs(diag[0] + diag[2] - (1 - 2 * p / 3)) < 1e-10
    assert abs(diag[1] + diag[3] - 2 * p / 3) < 1e-10


def test_dm_of_pure_circuit_matches_statevector(oracle):
    """tests/density_matrix.rs:131-180: DM diagonal == |psi|^2 for unitary circuits."""
    n = 4
    gates = oracle.brickwork(n, 3, 9)
    sv = oracle.simulate(n, gates)
    rho = oracle.dm_zero(n)
    for m, q in gates:
        oracle.dm_apply_channel(rho, n, [m], [1.0], q)
    assert np.max(np.abs(oracle.dm_populations(rho, n) - np.abs(sv) ** 2)) < 1e-10


def test_snap_rule(oracle):
    """cuda_gen.cpp:84-103: tolerances divided by K = 2^k."""
    m = np.array([[1 + 1e-13, 3e-13], [-1 + 2e-13j, 0.3]], dtype=complex)
    s = oracle.snap(m, 1e-12, 1e-12)  # K = 2: thresholds 5e-13
    assert s[0, 0] == 1 and s[0, 1] == 0 and s[1, 0] == -1 and s[1, 1] == 0.3
    m2 = np.array([[6e-13, 0], [0, 1]], dtype=complex)
    assert oracle.snap(m2, 1e-12, 1e-12)[0, 0] == 6e-13  # above ztol / K


def test_brickwork_structure(oracle):
    gates = oracle.brickwork(30, 20, 1)
    assert sum(1 for _, q in gates if len(q) == 1) == 600
    assert sum(1 for _, q in gates if len(q) == 2) == 290
