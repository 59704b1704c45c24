"""OpenQASM 2.0 front end on the GPU path (the reference parser's language,
src/openqasm/parser.rs:58-470): text -> parse_qasm -> circuit graph -> fusion
-> Simulator on the device, against the golden amplitudes derived from the
reference's tests/assets/qft_14.qasm and against the oracle."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("prec,fusion_k", [("f64", None), ("f64", 4), ("f32", 4)])
def test_qft14_qasm_text_on_gpu_matches_reference_fixture(cblib, oracle, prec, fusion_k):
    """The QFT-CX(14) circuit as OpenQASM text with the fixture's header
    (``OPENQASM 2.0; include "qelib1.inc"; qreg q[14];``), parsed, optionally
    fused, and simulated on the GPU from the reference test's seeded input
    (tests/cpu_cuda_compare.rs:54-69) reproduces the golden amplitudes:
    1e-10 per amplitude in FP64, 1e-5 in FP32 (cpu_cuda_compare.rs:27, 397)."""
    from cast_simulator_b200 import qasm
    from cast_simulator_b200.fusion import CircuitGraph, FusionConfig, optimize
    from cast_simulator_b200.simulator import Simulator
    from cast_simulator_b200.types import QuantumCircuit

    meta = json.load(open(os.path.join(GOLDEN, "qft14_meta.json")))
    text = qasm.to_qasm(QuantumCircuit.qft_cx(14))
    assert text.lstrip().startswith("OPENQASM 2.0;") and "qreg q[14];" in text
    circ = qasm.parse_qasm(text)
    assert circ.n_qubits() == meta["n_qubits"]
    graph = CircuitGraph.from_circuit(circ)
    if fusion_k is not None:
        optimize(graph, FusionConfig.size_only(fusion_k))
        assert len(graph.gates_in_row_order()) < len(circ.gates())
    sim = Simulator.f64() if prec == "f64" else Simulator.f32()
    got = sim.simulate(graph, initial=oracle.seeded_state(14)).download_amplitudes()
    golden = np.load(os.path.join(GOLDEN, "qft14_seeded.npy"))
    tol = 1e-10 if prec == "f64" else 1e-5
    assert np.max(np.abs(got - golden)) < tol


def test_handwritten_qasm_grammar_on_gpu(cblib, oracle):
    """Every statement form of the grammar (all named gates, angle expressions,
    the three operand spellings, comments) in one program, run on the GPU
    against the oracle applying the parsed gates."""
    from cast_simulator_b200 import qasm
    from cast_simulator_b200.fusion import CircuitGraph
    from cast_simulator_b200.simulator import Simulator

    text = """OPENQASM 2.0;
include "qelib1.inc";
qreg q[9];   // nine qubits
h q[0]; x q[1]; y q2; z 3; s q[4]; t q[5];
cx q[0], q[8]; cz q[1],q[7]; swap q[2], q[6];
ccx q[3], q[5], q[8];
rx(pi/3) q[0]; ry(-pi/7) q[4]; rz(2^3*pi/16) q[8];
cp(-(1+2)*pi/5) q[7], q[1];
u3(0.25, 1.5e-1, -pi) q[6];
u3(pi/2, 0, pi) q[3];
"""
    circ = qasm.parse_qasm(text)
    assert circ.n_qubits() == 9 and len(circ.gates()) == 16
    init = oracle.random_state(9, 21)
    ref = oracle.simulate(9, [(g.matrix(), g.qubits()) for g in circ.gates()], init)
    got = Simulator.f64().simulate(CircuitGraph.from_circuit(circ), initial=init).download_amplitudes()
    assert np.max(np.abs(got - ref)) < 1e-12
