"""The benchmark configurations at their specified sizes where the oracle can
follow: the 22-qubit QFT-CX on a seeded random complex128 state with the
default fusion against the oracle's FP64 run (the reference compares its CUDA
output with its CPU FP64 run, tests/cpu_cuda_compare.rs), and the brickwork
construction's size-independent properties at 24 qubits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.timeout(900)
def test_qft22_default_fusion_vs_oracle(cblib, oracle):
    from cast_simulator_b200.fusion import CircuitGraph, FusionConfig, optimize_native
    from cast_simulator_b200.simulator import Simulator
    from cast_simulator_b200.types import QuantumCircuit

    n = 22
    init = oracle.random_state(n, 2024)
    # the oracle runs the controlled-phase form (264 gates); it equals the
    # CX decomposition to 1e-12 (tests/test_oracle.py::test_qft_cx_equals_qft_cp)
    ref = oracle.simulate(n, oracle.qft_cp(n, True), init)
    circ = QuantumCircuit.qft_cx(n)
    fused = optimize_native(n, circ.gates(), FusionConfig.default()).gates()
    assert len(fused) < len(circ)
    got = Simulator.f64().simulate(CircuitGraph.from_gates(n, fused), initial=init).download_amplitudes()
    rep = oracle.fidelity_report(ref, got)
    assert rep["max_abs_err"] < 1e-10 and rep["one_minus_abs_overlap"] < 1e-12, rep


def test_brickwork24_fusion_widths_agree(cblib):
    """Every fusion width gives the same complex128 state, and a unit norm."""
    from cast_simulator_b200.fusion import CircuitGraph, FusionConfig, optimize_native
    from cast_simulator_b200.simulator import Simulator
    from cast_simulator_b200.types import QuantumCircuit

    n = 24
    circ = QuantumCircuit.brickwork(n, 20, 2024)
    outs = []
    for k in (2, 4, 6):
        fused = optimize_native(n, circ.gates(), FusionConfig.size_only(k)).gates()
        st = Simulator.f64().simulate(CircuitGraph.from_gates(n, fused))
        outs.append(st.download_amplitudes())
        assert abs(st.sv.norm_squared() - 1.0) < 1e-12
    assert np.max(np.abs(outs[0] - outs[1])) < 1e-12
    assert np.max(np.abs(outs[0] - outs[2])) < 1e-12
