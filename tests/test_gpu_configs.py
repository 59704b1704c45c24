"""The benchmark configurations at their specified sizes against the oracle
(the reference compares its CUDA output with its CPU FP64 run,
tests/cpu_cuda_compare.rs): the 22-qubit QFT-CX on a seeded random complex128
state with the default fusion, and the 30-qubit depth-20 brickwork - the
headline configuration, in complex128 and complex64 - against the threaded FP64
CPU restatement holding the full 16 GiB state on the host; plus the
construction's size-independent properties (fusion-width invariance, and the
circuit followed by its inverse returning to |0...0>)."""
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


def _compare_chunked(ref_state, sv, chunk_bits=24):
    """1 - |<ref|psi>| (psi renormalised) and max |ref - psi| over the whole
    state, reading both sides 2^chunk_bits amplitudes at a time (the device side
    through cast_cuda_sv_download at an offset pointer), so the host holds the
    FP64 reference plus two chunks."""
    from cast_simulator_b200 import _lib as L

    n = sv.n_qubits()
    prec = int(sv.precision())
    scalar = 8 if prec == 1 else 4
    cnt = 1 << min(chunk_bits, n)
    dot, nr, ng, err = 0j, 0.0, 0.0, 0.0
    eb = L.errbuf()
    buf = np.empty(cnt, dtype=np.complex128)
    for first in range(0, 1 << n, cnt):
        ref = ref_state.chunk(first, cnt)
        L.check(L.lib().cast_cuda_sv_download(sv.dptr + 2 * scalar * first,
                                              buf.view(np.float64).ctypes.data_as(L.c_dp), 2 * cnt,
                                              prec, eb, L.ERR_LEN), eb, "sv_download")
        dot += np.vdot(ref, buf)
        nr += float(np.vdot(ref, ref).real)
        ng += float(np.vdot(buf, buf).real)
        err = max(err, float(np.max(np.abs(ref - buf))))
    return 1.0 - abs(dot) / np.sqrt(nr * ng), err, ng


@pytest.mark.timeout(1800)
def test_brickwork30_headline_config_vs_cpu_oracle(cblib, oracle):
    """30 qubits, depth 20, fused at k = 4 (the benchmark's headline run) from
    |0...0>: the FP64 GPU state within 1e-10 per amplitude and 1 - |<>| <= 1e-12
    of the threaded FP64 CPU restatement, the FP32 GPU state within 1e-5 per
    amplitude and 1 - |<>| <= 1e-5 (tests/cpu_cuda_compare.rs:27, 397)."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.simulator import GateProgram, Stream
    from cast_simulator_b200.types import QuantumCircuit

    n = 30
    circ = QuantumCircuit.brickwork(n, 20, 2024)
    fused = optimize_native(n, circ.gates(), FusionConfig.size_only(4)).gates()
    assert len(circ) == 890 and len(fused) < 100
    with oracle.ThreadedState(n) as ref:
        ref.apply([(g.matrix(), g.qubits()) for g in fused])
        st = Stream()
        for prec, tol_amp, tol_ov in ((cu.CudaPrecision.F64, 1e-10, 1e-12),
                                      (cu.CudaPrecision.F32, 1e-5, 1e-5)):
            tol = 1e-12 if prec == cu.CudaPrecision.F64 else 1e-6
            prog = GateProgram(prec, n, tol, tol)
            for g in fused:
                prog.add(g.matrix(), g.qubits())
            sv = cu.CudaStatevector(n, prec)
            sv.zero(st)
            prog.run(sv, st, use_graph=False)
            st.sync()
            one_minus, err, norm2 = _compare_chunked(ref, sv)
            assert err < tol_amp and one_minus < tol_ov, (prec, err, one_minus)
            assert abs(norm2 - 1.0) < (1e-12 if prec == cu.CudaPrecision.F64 else 1e-5)
            del sv, prog


@pytest.mark.timeout(600)
def test_brickwork30_then_inverse_returns_to_zero(cblib):
    """A size-independent property at the full size: the fused 30-qubit circuit
    followed by its inverse (the fused gates' adjoints in reverse order) maps
    |0...0> back to |0...0>: amplitude 0 within 1e-12 of 1 (complex128), and the
    norm stays 1."""
    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.simulator import GateProgram, Stream
    from cast_simulator_b200.types import QuantumCircuit

    n = 30
    circ = QuantumCircuit.brickwork(n, 20, 2024)
    fused = optimize_native(n, circ.gates(), FusionConfig.size_only(4)).gates()
    prog = GateProgram(cu.CudaPrecision.F64, n, 1e-12, 1e-12)
    for g in fused:
        prog.add(g.matrix(), g.qubits())
    for g in reversed(fused):
        prog.add(np.conj(g.matrix()).T, g.qubits())
    sv = cu.CudaStatevector(n, cu.CudaPrecision.F64)
    st = Stream()
    sv.zero(st)
    prog.run(sv, st, use_graph=False)
    st.sync()
    a0 = np.zeros(2)
    eb = L.errbuf()
    L.check(L.lib().cast_cuda_sv_download(sv.dptr, a0.ctypes.data_as(L.c_dp), 2, 1, eb, L.ERR_LEN),
            eb, "sv_download")
    assert abs(a0[0] - 1.0) < 1e-12 and abs(a0[1]) < 1e-12, a0
    assert abs(sv.norm_squared() - 1.0) < 1e-12
