"""Split-BF16 tensor-core path (complex64, fused gates with 5 or 6 qubits).

Stated bound, per fused pass: every amplitude within 1e-4 of the largest
reference amplitude (relative product error ~2^-16), a direction error
1 - |<ref|psi>| / ||psi|| <= 1e-8 and a norm drift |1 - ||psi||| <= 2^-16.  The
split operands perturb each product by ~2^-17 relative; the component of that
perturbation along psi changes the norm linearly (~1e-6 on a single 64-amplitude
group, less when many groups average), while the perpendicular component only
enters the direction error quadratically (~1e-11).  A whole fused circuit,
renormalised at the end, stays within 1 - |<ref|psi>| <= 1e-6 of the FP64
oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cblib):
    from cast_simulator_b200 import cuda, fusion, simulator, types

    return cuda, fusion, simulator, types


def haar(rng, d):
    z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _cases(rng, k):
    """(n, qubits): high, low and mixed placements on 16 qubits; a partial tile
    (fewer than 128 groups) and a statevector of exactly the gate's qubits."""
    n = 16
    out = [(n, tuple(range(n - k, n))), (n, tuple(range(k))),
           (n, tuple(sorted([0, 3] + list(range(n - k + 2, n))))),
           (n, tuple(sorted(rng.choice(n, size=k, replace=False).tolist())))]
    out += [(k + 3, tuple(range(1, k + 1))), (k, tuple(range(k)))]
    # lowest target 5, 7 and 9: register loads, then the TMA-fed kernel (1 KB runs)
    out += [(n, tuple([5] + list(range(n - k + 1, n)))), (n, tuple(range(7, 7 + k))),
            (n, tuple(range(9, 9 + k)))]
    if k == 5:
        # a 5-qubit gate runs padded to 6 qubits with the identity on a spare qubit:
        # no spare >= 7 (the highest free qubit is used), and the padded gate
        # filling the whole statevector
        out += [(10, (2, 6, 7, 8, 9)), (6, (0, 1, 2, 3, 4)), (6, (1, 2, 3, 4, 5))]
    return out


@pytest.mark.parametrize("loader", [0, 2])
@pytest.mark.parametrize("k", [5, 6])
def test_single_gate_within_bound(mods, oracle, k, loader):
    """loader 0: register loads everywhere (the default); loader 2: TMA bulk
    copies where eligible (lowest target >= 7, whole tiles), register loads
    otherwise."""
    cu, F, S, T = mods
    from cast_simulator_b200 import _lib as L

    rng = np.random.default_rng(40 + k)
    S.tensor_status()  # clear the error word
    old = L.lib().cast_b200_set_tensor_loader(loader)
    try:
        _check_cases(cu, S, oracle, k, _cases(rng, k), rng)
    finally:
        L.lib().cast_b200_set_tensor_loader(old)


def _check_cases(cu, S, oracle, k, cases, rng):
    for n, q in cases:
        m = haar(rng, 1 << k)
        init = oracle.random_state(n, k)
        ref = init.copy()
        oracle.apply_gate(ref, m, q)
        prog = S.GateProgram(cu.CudaPrecision.F32, n, 1e-6, 1e-6, split_precision=True)
        prog.add(m, q)
        sv = cu.CudaStatevector(n, cu.CudaPrecision.F32)
        sv.upload(init)
        st = S.Stream()
        prog.run(sv, st, use_graph=False)
        st.sync()
        got = sv.download()
        rep = oracle.fidelity_report(ref, got)
        nrm = float(np.linalg.norm(got))
        direction = 1.0 - abs(oracle.inner(ref, got)) / nrm
        print(f"k={k} q={q} max_err={rep['max_abs_err']:.3e} 1-|ov|={rep['one_minus_abs_overlap']:.3e} "
              f"direction={direction:.3e} norm_drift={1 - nrm:.3e}")
        assert S.tensor_status() == 0
        assert rep["max_abs_err"] <= 1e-4 * np.max(np.abs(ref)), (n, q, rep)
        assert direction <= 1e-8, (n, q, direction)
        assert abs(1.0 - nrm) <= 2.0 ** -16, (n, q, nrm)


@pytest.mark.parametrize("k", [4, 5, 6])
def test_fused_circuit_fidelity(mods, oracle, k):
    cu, F, S, T = mods
    n = 20
    circ = T.QuantumCircuit.brickwork(n, 12, 77)
    ref = oracle.simulate(n, [(g.matrix(), g.qubits()) for g in circ.gates()])
    fused = F.optimize_native(n, circ.gates(), F.FusionConfig.size_only(k)).gates()
    assert max(g.n_qubits() for g in fused) == k
    sim = S.Simulator(cu.CudaKernelGenSpec.f32(), split_precision=True)
    state = sim.simulate(F.CircuitGraph.from_gates(n, fused))
    raw = state.download_amplitudes()
    state.sv.normalize()
    got = state.download_amplitudes()
    rep = oracle.fidelity_report(ref, got)
    print(f"k={k} circuit: 1-|ov| renormalised={rep['one_minus_abs_overlap']:.3e} "
          f"raw={oracle.fidelity_report(ref, raw)['one_minus_abs_overlap']:.3e}")
    assert S.tensor_status() == 0
    assert rep["one_minus_abs_overlap"] <= 1e-6, rep
    plain = S.Simulator(cu.CudaKernelGenSpec.f32()).simulate(F.CircuitGraph.from_gates(n, fused))
    rep_plain = oracle.fidelity_report(ref, plain.download_amplitudes())
    assert rep_plain["one_minus_abs_overlap"] <= 1e-6


def test_split_mode_keeps_small_gates_on_cuda_cores(mods, oracle):
    """Gates below 5 qubits in a split-precision program run on the FP32 CUDA-core
    kernels (FP32 accuracy, not the split-BF16 bound)."""
    cu, F, S, T = mods
    rng = np.random.default_rng(9)
    n = 14
    for k in (1, 2, 3, 4):
        q = tuple(sorted(rng.choice(n, size=k, replace=False).tolist()))
        m = haar(rng, 1 << k)
        init = oracle.random_state(n, 3)
        ref = init.copy()
        oracle.apply_gate(ref, m, q)
        prog = S.GateProgram(cu.CudaPrecision.F32, n, 1e-6, 1e-6, split_precision=True)
        prog.add(m, q)
        sv = cu.CudaStatevector(n, cu.CudaPrecision.F32)
        sv.upload(init)
        st = S.Stream()
        prog.run(sv, st, use_graph=False)
        st.sync()
        assert np.max(np.abs(sv.download() - ref)) < 1e-6, (k, q)


def test_split_mode_must_precede_gates(mods):
    cu, F, S, T = mods
    prog = S.GateProgram(cu.CudaPrecision.F32, 8, 1e-6, 1e-6)
    prog.add(np.eye(2), (0,))
    from cast_simulator_b200 import _lib as L

    eb = L.errbuf()
    assert L.lib().cast_b200_program_set_split_precision(prog.handle, 1, eb, L.ERR_LEN) == 1
    assert b"before adding gates" in eb.value
