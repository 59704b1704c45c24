"""OpenQASM 2.0 front-end (the reference parser's language, src/openqasm/
parser.rs:58-470, and its tests at parser.rs:828+), pinned end to end against
the golden vectors derived from the reference's tests/assets/qft_14.qasm."""
import json
import math
import os

import numpy as np
import pytest

from cast_simulator_b200 import qasm
from cast_simulator_b200.types import QuantumCircuit, QuantumGate

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_program_without_qreg_declaration():
    c = qasm.parse_qasm("h q[0];\ncx q[0], q[2];")
    assert c.n_qubits() == 3 and len(c.gates()) == 2


def test_preamble_and_qreg():
    c = qasm.parse_qasm('OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg q[4]; // four qubits\nx q[3];')
    assert c.n_qubits() == 4
    assert np.array_equal(c.gates()[0].matrix(), QuantumGate.x(3).matrix())


def test_parametric_gates_and_angles():
    c = qasm.parse_qasm("qreg q[3]; rz(pi/2) q[0]; rx(-pi/4) q1; u3(2^3*pi/16, (1+2)*pi, -.5) 2;"
                        " cp(pi^2/pi) q[0],q[2]; ry(1.5e-1) q[1];")
    g = c.gates()
    assert np.allclose(g[0].matrix(), QuantumGate.rz(math.pi / 2, 0).matrix(), atol=0)
    assert np.allclose(g[1].matrix(), QuantumGate.rx(-math.pi / 4, 1).matrix(), atol=0)
    assert np.allclose(g[2].matrix(), QuantumGate.u3(8 * math.pi / 16, 3 * math.pi, -0.5, 2).matrix(), atol=0)
    assert np.allclose(g[3].matrix(), QuantumGate.cp(math.pi, 0, 2).matrix(), atol=1e-15)
    assert g[4].op() == ("ry", (0.15,), (1,))
    # control/target order survives canonicalisation: cx 2,0 is not cx 0,2
    a, b = qasm.parse_qasm("cx q[2],q[0]; cx q[0],q[2];").gates()
    assert a.qubits() == b.qubits() == (0, 2) and not np.array_equal(a.matrix(), b.matrix())


@pytest.mark.parametrize("text,msg", [
    ("qreg q[2]; h q[2];", "out of bounds"),
    ("qreg q[2]; h r[0];", "unknown qreg"),
    ("qreg q[2]; qreg r[2];", "multiple qreg"),
    ("foo q[0];", "unsupported gate"),
    ("h q[0]", "expected `;`"),
    ("rz(pi/) q[0];", "expected expression term"),
    ("h q[0]; $", "unsupported character"),
    ("OPENQASM 2.0", "end-of-input"),
])
def test_errors(text, msg):
    with pytest.raises(ValueError, match=msg):
        qasm.parse_qasm(text)


def test_qft14_round_trip_matches_reference_fixture(oracle):
    """QFT-CX(14) written as OpenQASM, parsed back and simulated reproduces the
    golden amplitudes of the reference's qft_14.qasm on its seeded input."""
    meta = json.load(open(os.path.join(GOLDEN, "qft14_meta.json")))
    text = qasm.to_qasm(QuantumCircuit.qft_cx(14))
    circ = qasm.parse_qasm(text)
    counts = {}
    for g in circ.gates():
        counts[g.op()[0]] = counts.get(g.op()[0], 0) + 1
    assert counts == meta["gate_counts"] and circ.n_qubits() == meta["n_qubits"]
    out = oracle.simulate(14, [(g.matrix(), g.qubits()) for g in circ.gates()], oracle.seeded_state(14))
    assert np.max(np.abs(out - np.load(os.path.join(GOLDEN, "qft14_seeded.npy")))) < 1e-12
    with pytest.raises(ValueError, match="named standard gates"):
        c = QuantumCircuit(2)
        c.add(QuantumGate.h(0).matmul(QuantumGate.x(1)))
        qasm.to_qasm(c)
