"""The trajectory-program builder on the host, without a GPU: channel
classification, and the exactness of the program it emits.  Pauli errors
inside a fused block are moved to the block's end as U_s P U_s^dagger (U_s the
block's gates after the error), damping on consecutive qubits is merged into
one mask, other one-qubit channels stay general.  The emitted program, read as
a sequence of channels, must give exactly the density matrix of the original
circuit (both evolved with the CPU oracle)."""
import math

import numpy as np
import pytest

from cast_simulator_b200 import trajectory as TR
from cast_simulator_b200.types import QuantumCircuit, QuantumGate, mat_x, mat_y, mat_z


def test_channel_classification():
    p, mats = TR._is_pauli_channel(QuantumGate.depolarizing(3, 0.03))
    assert p == pytest.approx(0.03) and len(mats) == 3
    p, mats = TR._is_pauli_channel(QuantumGate.bit_flip(0, 0.1))
    assert p == pytest.approx(0.1) and all(np.allclose(m, mat_x()) for m in mats)
    p, mats = TR._is_pauli_channel(QuantumGate.phase_flip(0, 0.2))
    assert p == pytest.approx(0.2) and all(np.allclose(m, mat_z()) for m in mats)
    assert TR._is_pauli_channel(QuantumGate.pauli_channel(0, 0.1, 0.05, 0.2)) is None
    assert TR._is_pauli_channel(QuantumGate.amplitude_damping(0, 0.1)) is None
    assert TR._is_pauli_channel(QuantumGate.h(0)) is None
    assert TR._damping_rate(QuantumGate.amplitude_damping(2, 0.125)) == pytest.approx(0.125)
    assert TR._damping_rate(QuantumGate.depolarizing(2, 0.1)) is None
    assert TR._damping_rate(QuantumGate.phase_flip(2, 0.1)) is None


def _circuit():
    c = QuantumCircuit(4)
    c.add(QuantumGate.h(0))
    c.add(QuantumGate.depolarizing(0, 0.05))
    c.add(QuantumGate.cx(0, 1))
    c.add(QuantumGate.depolarizing(0, 0.1))
    c.add(QuantumGate.depolarizing(1, 0.07))
    c.add(QuantumGate.u3(0.7, 0.2, -0.4, 2))
    c.add(QuantumGate.depolarizing(2, 0.02))
    c.add(QuantumGate.cz(2, 3))
    c.add(QuantumGate.bit_flip(3, 0.1))
    c.add(QuantumGate.u3(1.1, -0.3, 0.5, 3))
    for q in range(4):
        c.add(QuantumGate.amplitude_damping(q, 0.1))
    c.add(QuantumGate.pauli_channel(1, 0.1, 0.05, 0.2))
    c.add(QuantumGate.u3(0.3, 0.9, 0.1, 1))
    c.add(QuantumGate.cx(1, 2))
    c.add(QuantumGate.phase_flip(1, 0.03))
    return c


def _record(monkeypatch):
    ops = []
    monkeypatch.setattr(TR.TrajectoryProgram, "_add_gate",
                        lambda self, m, q: ops.append(("gate", np.array(m), tuple(q))))
    monkeypatch.setattr(TR.TrajectoryProgram, "_add_error",
                        lambda self, p, mats: ops.append(("err", p, [np.array(x) for x in mats])))
    monkeypatch.setattr(TR.TrajectoryProgram, "_add_damping",
                        lambda self, mask, g: ops.append(("damp", mask, g)))
    monkeypatch.setattr(TR.TrajectoryProgram, "_add_channel",
                        lambda self, q, kraus: ops.append(("chan", q, [np.array(x) for x in kraus])))
    return ops


@pytest.mark.parametrize("fusion_k", [1, 2, 3, 4])
def test_program_equals_circuit_as_channels(monkeypatch, oracle, cblib, fusion_k):
    ops = _record(monkeypatch)
    circ = _circuit()
    TR.TrajectoryProgram(circ, fusion_k, native=False)  # the Python builder, recorded
    n = circ.n_qubits()
    # the reference: every gate / channel of the circuit, in order
    ref = oracle.dm_zero(n)
    for g in circ.gates():
        if g.is_unitary():
            oracle.dm_apply_channel(ref, n, [g.matrix()], [1.0], g.qubits())
        else:
            br = g.noise_model().branches
            oracle.dm_apply_channel(ref, n, [k for _, k in br], [p for p, _ in br], g.qubits())
    # the program read as channels: errors act on the block before them
    rho = oracle.dm_zero(n)
    block_q = None
    kinds = [o[0] for o in ops]
    for op in ops:
        if op[0] == "gate":
            _, m, q = op
            block_q = q
            oracle.dm_apply_channel(rho, n, [m], [1.0], q)
        elif op[0] == "err":
            _, p, mats = op
            d = 1 << len(block_q)
            oracle.dm_apply_channel(rho, n, [np.eye(d)] + mats, [1 - p] + [p / 3] * 3, block_q)
        elif op[0] == "damp":
            _, mask, g = op
            k0 = np.diag([1.0, math.sqrt(1 - g)])
            k1 = np.array([[0.0, math.sqrt(g)], [0.0, 0.0]])
            for q in range(n):
                if (mask >> q) & 1:
                    oracle.dm_apply_channel(rho, n, [k0, k1], [1.0, 1.0], (q,))
        else:
            _, q, kraus = op
            oracle.dm_apply_channel(rho, n, kraus, [1.0] * len(kraus), (q,))
    assert np.max(np.abs(rho - ref)) < 1e-12
    # the four damping sites merge into one mask; the unequal Pauli channel stays general
    assert [o for o in ops if o[0] == "damp"] == [("damp", 0b1111, pytest.approx(0.1))]
    assert kinds.count("chan") == 1
    assert kinds.count("err") == 6  # one per Pauli site


def _dm_of_ops(oracle, n, ops):
    """Density matrix of a trajectory program read as a channel sequence
    (ops as TrajectoryProgram.ops() returns them)."""
    rho = oracle.dm_zero(n)
    block_q = None
    for kind, k, q, p, mask, mats in ops:
        if kind == "gate":
            block_q = q
            oracle.dm_apply_channel(rho, n, mats, [1.0], q)
        elif kind == "err":
            d = 1 << len(block_q)
            oracle.dm_apply_channel(rho, n, [np.eye(d)] + mats, [1 - p] + [p / 3] * 3, block_q)
        elif kind == "damp":
            k0 = np.diag([1.0, math.sqrt(1 - p)])
            k1 = np.array([[0.0, math.sqrt(p)], [0.0, 0.0]])
            for qq in range(n):
                if (mask >> qq) & 1:
                    oracle.dm_apply_channel(rho, n, [k0, k1], [1.0, 1.0], (qq,))
        else:
            oracle.dm_apply_channel(rho, n, mats, [1.0] * len(mats), q)
    return rho


@pytest.mark.parametrize("fusion_k", [1, 2, 3, 4])
def test_native_builder_equals_python_builder(oracle, cblib, fusion_k):
    """The native builder (cast_b200_traj_build) emits the Python builder's
    program: same op sequence, qubits and probabilities, matrices equal to the
    complex64 storage precision; read as channels it reproduces the circuit's
    density matrix."""
    circ = _circuit()
    n = circ.n_qubits()
    nat = TR.TrajectoryProgram(circ, fusion_k, native=True)
    py = TR.TrajectoryProgram(circ, fusion_k, native=False)
    a, b = nat.ops(), py.ops()
    assert [(o[0], o[1], o[2], o[4]) for o in a] == [(o[0], o[1], o[2], o[4]) for o in b]
    for x, y in zip(a, b):
        assert x[3] == pytest.approx(y[3], abs=1e-7)
        assert all(np.max(np.abs(mx - my)) < 1e-6 for mx, my in zip(x[5], y[5]))
    assert (nat.stats.n_blocks, nat.stats.n_errors, nat.stats.n_damping, nat.stats.n_channels) == \
        (py.stats.n_blocks, py.stats.n_errors, py.stats.n_damping, py.stats.n_channels)
    ref = oracle.dm_zero(n)
    for g in circ.gates():
        if g.is_unitary():
            oracle.dm_apply_channel(ref, n, [g.matrix()], [1.0], g.qubits())
        else:
            br = g.noise_model().branches
            oracle.dm_apply_channel(ref, n, [k for _, k in br], [p for p, _ in br], g.qubits())
    assert np.max(np.abs(_dm_of_ops(oracle, n, a) - ref)) < 1e-5


def test_native_builder_brickwork_matches_python(cblib):
    """The trajectory configuration's construction (brickwork, depolarizing after
    every gate, damping every layer) at 12 qubits builds the same program both ways."""
    circ = QuantumCircuit.brickwork(12, 6, 5, depolarizing=1e-3, damping=5e-4)
    a = TR.TrajectoryProgram(circ, 3, native=True).ops()
    b = TR.TrajectoryProgram(circ, 3, native=False).ops()
    assert len(a) == len(b) > 0
    assert [(o[0], o[2], o[4]) for o in a] == [(o[0], o[2], o[4]) for o in b]
    assert max(np.max(np.abs(mx - my)) for x, y in zip(a, b) for mx, my in zip(x[5], y[5])) < 1e-6


def test_native_builder_rejects_wide_channels(cblib):
    c = QuantumCircuit(3)
    c.add(QuantumGate.cx(0, 1).with_noise([(0.99, np.eye(4)), (0.01, np.kron(mat_x(), np.eye(2)))]))
    with pytest.raises(ValueError, match="single-qubit channels"):
        TR.TrajectoryProgram(c, 3)
