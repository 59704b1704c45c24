"""The native C++ fusion planner makes the same decisions as the host-side
mirror of fusion.rs / circuit_graph.rs (and both preserve the circuit)."""
import time

import numpy as np
import pytest

from cast_simulator_b200 import fusion as F
from cast_simulator_b200.types import QuantumCircuit, QuantumGate


def _cases():
    rng = np.random.default_rng(4)
    rand = QuantumCircuit(9)
    for _ in range(60):
        k = int(rng.integers(1, 4))
        q = sorted(rng.choice(9, size=k, replace=False).tolist())
        rand.add(QuantumGate.random_unitary(q, rng))
    return [QuantumCircuit.brickwork(12, 8, 3), QuantumCircuit.qft_cx(10), QuantumCircuit.qft(9),
            rand]


@pytest.mark.parametrize("k", [2, 3, 4, 5, 6, 7])
def test_native_matches_python_size_only(cblib, k):
    for circ in _cases():
        g = F.CircuitGraph.from_circuit(circ)
        F.optimize(g, F.FusionConfig.size_only(k))
        py = g.gates_in_row_order()
        nat = F.optimize_native(circ.n_qubits(), circ.gates(), F.FusionConfig.size_only(k)).gates()
        assert len(py) == len(nat)
        for a, b in zip(py, nat):
            assert a.qubits() == b.qubits()
            assert np.max(np.abs(a.matrix() - b.matrix())) < 1e-12


def test_native_matches_python_hardware_adaptive(cblib):
    prof = F.HardwareProfile.from_roofline({"device": "test"}, 3000.0, 2000.0, 8)
    prof.tensor_gflops_s, prof.tensor_min_k = 20000.0, 5
    cfg = F.FusionConfig.hardware_adaptive(prof, 7, 1e-12)
    for circ in _cases():
        g = F.CircuitGraph.from_circuit(circ)
        F.optimize(g, cfg)
        py = g.gates_in_row_order()
        nat = F.optimize_native(circ.n_qubits(), circ.gates(), cfg).gates()
        assert [x.qubits() for x in py] == [x.qubits() for x in nat]


def test_native_is_fast_and_preserves_the_circuit(cblib, oracle):
    circ = QuantumCircuit.brickwork(28, 40, 9)
    t = time.perf_counter()
    fused = F.optimize_native(28, circ.gates(), F.FusionConfig.size_only(4))
    assert time.perf_counter() - t < 2.0 and 0 < len(fused) < len(circ)
    small = QuantumCircuit.brickwork(10, 12, 1)
    ref = oracle.simulate(10, [(g.matrix(), g.qubits()) for g in small.gates()])
    out = oracle.simulate(10, [(g.matrix(), g.qubits()) for g in
                               F.optimize_native(10, small.gates(), F.FusionConfig.size_only(5)).gates()])
    assert np.max(np.abs(out - ref)) < 1e-12


def test_native_rejects_bad_input(cblib):
    with pytest.raises(Exception, match="size_max"):
        F.optimize_native(4, [QuantumGate.h(0)], F.FusionConfig.size_only(9))
