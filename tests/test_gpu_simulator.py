"""GPU tests of the Simulator API, gate programs (CUDA graphs), fusion on the
device path, both kernel paths, reductions and the density-matrix mode."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cblib):
    from cast_simulator_b200 import _lib, cuda, fusion, simulator, types

    return _lib, cuda, fusion, simulator, types


def _oracle_gates(circ):
    return [(g.matrix(), g.qubits()) for g in circ.gates()]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("k", [2, 3, 4, 5, 6, 7])
def test_fused_brickwork_matches_unfused_oracle(mods, oracle, prec, k):
    """Fusion invariance through the GPU path (tests/fusion_correctness.rs)."""
    L, cu, F, S, T = mods
    n = 14
    circ = T.QuantumCircuit.brickwork(n, 8, 11)
    ref = oracle.simulate(n, _oracle_gates(circ))
    g = F.CircuitGraph.from_circuit(circ)
    F.optimize(g, F.FusionConfig.size_only(k))
    sim = S.Simulator.f64() if prec == "f64" else S.Simulator.f32()
    got = sim.simulate(g).download_amplitudes()
    rep = oracle.fidelity_report(ref, got)
    if prec == "f64":
        assert rep["max_abs_err"] < 1e-10 and rep["one_minus_abs_overlap"] < 1e-12
    else:
        assert rep["max_abs_err"] < 1e-5 and rep["one_minus_abs_overlap"] < 1e-5


def test_qft_cx_program_graph_and_eager(mods, oracle):
    L, cu, F, S, T = mods
    n = 16
    circ = T.QuantumCircuit.qft_cx(n)
    init = oracle.random_state(n, 21)
    ref = oracle.simulate(n, _oracle_gates(circ), init)
    for use_graph in (True, False):
        sim = S.Simulator.f64()
        sim.use_graph = use_graph
        got = sim.simulate(F.CircuitGraph.from_circuit(circ), initial=init).download_amplitudes()
        assert np.max(np.abs(got - ref)) < 1e-10
    # replaying one program twice = applying the circuit twice
    prog = S.Simulator.f64().compile_batch(circ.gates(), n)
    sv = cu.CudaStatevector(n, cu.CudaPrecision.F64)
    sv.upload(init)
    st = S.Stream()
    prog.run(sv, st)
    prog.run(sv, st)
    st.sync()
    ref2 = oracle.simulate(n, _oracle_gates(circ), ref)
    assert np.max(np.abs(sv.download() - ref2)) < 1e-10


@pytest.mark.parametrize("path", [1, 2])
@pytest.mark.parametrize("prec", [1, 0])
def test_forced_kernel_paths(mods, oracle, path, prec):
    """Register and tile kernels agree with the oracle on every low-qubit pattern."""
    L, cu, F, S, T = mods
    lib = L.lib()
    old = lib.cast_b200_set_gate_path(path)
    try:
        rng = np.random.default_rng(5)
        n = 13
        for q in [(0, 1), (0, 2), (0, 1, 2), (1, 2, 12), (0, 1, 2, 3), (2, 3, 4), (0, 4, 9, 12), (3,)]:
            d = 1 << len(q)
            z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
            m = np.linalg.qr(z)[0]
            init = oracle.random_state(n, 3)
            ref = init.copy()
            oracle.apply_gate(ref, m, q)
            sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
            sv.upload(init)
            mm = np.ascontiguousarray(m)
            qq = np.asarray(q, dtype=np.uint32)
            eb = L.errbuf()
            tol = 1e-12 if prec else 1e-6
            L.check(lib.cast_b200_apply_gate(sv.dptr, n, prec, mm.view(np.float64).ctypes.data_as(
                C.POINTER(L.Complex64)), qq.ctypes.data_as(L.c_u32p), qq.size, tol, tol, None, eb,
                L.ERR_LEN), eb)
            got = sv.download()
            assert np.max(np.abs(got - ref)) < (1e-12 if prec else 1e-5), q
    finally:
        lib.cast_b200_set_gate_path(old)


@pytest.mark.parametrize("prec", [1, 0])
def test_kernel_choice_tile_sizes(mods, oracle, prec):
    """Each kernel a low-target class can be routed to (register, tile of 2048
    or 4096 amplitudes) agrees with the oracle."""
    L, cu, F, S, T = mods
    lib = L.lib()
    rng = np.random.default_rng(9)
    n = 14
    pats = [(0,), (4,), (0, 1), (1, 3), (0, 13), (0, 1, 2), (2, 4, 12), (0, 1, 2, 3), (1, 2, 3, 4),
            (0, 4, 9, 13), (3, 7, 12, 13)]
    try:
        for q in pats:
            d = 1 << len(q)
            z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
            m = np.linalg.qr(z)[0]
            mask = sum(1 << b for b in q if b < 5)
            init = oracle.random_state(n, 4)
            ref = init.copy()
            oracle.apply_gate(ref, m, q)
            for eng, tb in [("register", 0), ("tile", 11), ("tile", 12)]:
                S.set_kernel_choice(cu.CudaPrecision(prec), len(q), mask, eng, tb)
                assert S.gate_engine(m, q, n, cu.CudaPrecision(prec)) == eng
                sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
                sv.upload(init)
                prog = S.GateProgram(cu.CudaPrecision(prec), n, 1e-12, 1e-12)
                prog.add(m, q)
                prog.run(sv, None, use_graph=False)
                got = sv.download()
                assert np.max(np.abs(got - ref)) < (1e-12 if prec else 1e-5), (q, eng, tb)
            S.set_kernel_choice(cu.CudaPrecision(prec), len(q), mask, None)
    finally:
        for k in range(1, 5):
            for mask in range(1, 32):
                if bin(mask).count("1") <= k:
                    S.set_kernel_choice(cu.CudaPrecision(prec), k, mask, None)


def test_tune_kernels_small(mods):
    """The kernel autotuner runs over every class of a small register, returns a
    valid winner per class and leaves the built-in rule in place without apply."""
    from cast_simulator_b200 import autotune as A

    L, cu, F, S, T = mods
    recs = A.tune_kernels(14, ("f32",), ks=(2, 3), reps=1, apply=False)
    assert len(recs) == len(A.kernel_classes((2, 3)))
    rng = np.random.default_rng(1)
    for r in recs:
        assert (r["engine"], r["tile_bits"]) in A.KERNEL_CANDIDATES
        assert set(r["ms"]) == {"register", "tile11", "tile12"}
        assert all(v > 0 for v in r["ms"].values())
        d = 1 << r["k"]
        z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        assert S.gate_engine(np.linalg.qr(z)[0], tuple(r["targets"]), 14,
                             cu.CudaPrecision.F32) == r["builtin"]
    assert A.apply_kernel_choices(recs[:2]) == 2
    for r in recs[:2]:
        S.set_kernel_choice(cu.CudaPrecision.F32, r["k"], r["low_mask"], None)


def test_apply_gate_large_k_and_errors(mods, oracle):
    L, cu, F, S, T = mods
    lib = L.lib()
    rng = np.random.default_rng(8)
    n = 12
    for q in [(0, 1, 2, 3, 4, 5), (1, 3, 5, 7, 9, 10, 11)]:
        d = 1 << len(q)
        m = np.linalg.qr(rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d)))[0]
        init = oracle.random_state(n, 4)
        ref = init.copy()
        oracle.apply_gate(ref, m, q)
        sv = cu.CudaStatevector(n, cu.CudaPrecision.F64)
        sv.upload(init)
        qq = np.asarray(q, dtype=np.uint32)
        mm = np.ascontiguousarray(m)
        eb = L.errbuf()
        L.check(lib.cast_b200_apply_gate(sv.dptr, n, 1, mm.view(np.float64).ctypes.data_as(
            C.POINTER(L.Complex64)), qq.ctypes.data_as(L.c_u32p), qq.size, 1e-12, 1e-12, None, eb,
            L.ERR_LEN), eb)
        assert np.max(np.abs(sv.download() - ref)) < 1e-10
    eb = L.errbuf()
    qq = np.asarray([3, 12], dtype=np.uint32)
    mm = np.eye(4, dtype=np.complex128)
    rc = lib.cast_b200_apply_gate(sv.dptr, n, 1, mm.view(np.float64).ctypes.data_as(
        C.POINTER(L.Complex64)), qq.ctypes.data_as(L.c_u32p), 2, 0.0, 0.0, None, eb, L.ERR_LEN)
    assert rc == 1 and b"outside" in eb.value


@pytest.mark.parametrize("prec", [1, 0])
def test_reductions(mods, oracle, prec):
    L, cu, F, S, T = mods
    n = 17
    a = oracle.random_state(n, 1)
    b = oracle.random_state(n, 2)
    sa = cu.CudaStatevector(n, cu.CudaPrecision(prec))
    sb = cu.CudaStatevector(n, cu.CudaPrecision(prec))
    sa.upload(a)
    sb.upload(b)
    a_, b_ = sa.download(), sb.download()  # compare against the stored precision
    ip = S.inner_product(sa, sb)
    assert abs(ip - np.vdot(a_, b_)) < 1e-12
    p1, nrm = S.qubit_populations(sa)
    probs = np.abs(a_) ** 2
    idx = np.arange(1 << n)
    exp = np.array([probs[(idx >> q) & 1 == 1].sum() for q in range(n)])
    assert np.max(np.abs(p1 - exp)) < 1e-12 and abs(nrm - probs.sum()) < 1e-12
    meas = [0, 5, 16]
    mp = S.marginal_probabilities(sa, meas)
    bins = sum((((idx >> q) & 1) << j) for j, q in enumerate(meas))
    assert np.max(np.abs(mp - np.bincount(bins, weights=probs, minlength=8))) < 1e-12


def test_density_matrix_noisy_circuit(mods, oracle):
    """DM mode on the device vs the oracle's channel-by-channel evolution."""
    L, cu, F, S, T = mods
    n = 5
    circ = T.QuantumCircuit.brickwork(n, 3, 4, depolarizing=0.05, damping=0.1)
    rho = oracle.dm_zero(n)
    for g in circ.gates():
        if g.is_unitary():
            oracle.dm_apply_channel(rho, n, [g.matrix()], [1.0], g.qubits())
        else:
            br = g.noise_model().branches
            oracle.dm_apply_channel(rho, n, [k for _, k in br], [p for p, _ in br], g.qubits())
    ref = oracle.dm_populations(rho, n)
    graph = F.CircuitGraph.from_circuit(circ)
    state = S.Simulator.f64().simulate(graph, S.Representation.DensityMatrix)
    pops = state.populations()
    assert np.max(np.abs(pops - ref)) < 1e-10
    assert abs(state.trace() - 1.0) < 1e-10
    with pytest.raises(ValueError, match="non-unitary"):
        S.Simulator.f64().simulate(graph, S.Representation.StateVector)


def test_expectation_z_and_bench(mods, oracle):
    L, cu, F, S, T = mods
    n = 12
    circ = T.QuantumCircuit.brickwork(n, 5, 3)
    ref = oracle.simulate(n, _oracle_gates(circ))
    probs = np.abs(ref) ** 2
    idx = np.arange(1 << n)
    z_ref = np.array([1 - 2 * probs[(idx >> q) & 1 == 1].sum() for q in range(n)])
    sim = S.Simulator.f64()
    graph = F.CircuitGraph.from_circuit(circ)
    z = sim.simulate(graph).expectation_z()
    assert np.max(np.abs(z - z_ref)) < 1e-12
    rt = sim.bench(graph, budget_s=0.05)
    assert rt.exec.n_iters() >= 3 if hasattr(rt.exec, "n_iters") else len(rt.exec.samples_s) >= 3


def test_simulate_reuses_statevector_memory(mods, oracle):
    """A dropped QuantumState hands its allocation back to the Simulator; the
    next simulate of the same width reuses it (no 2^n-sized cudaMalloc per call)
    and the results are unaffected."""
    L, cu, F, S, T = mods
    n = 14
    circ = T.QuantumCircuit.brickwork(n, 6, 21)
    ref = oracle.simulate(n, _oracle_gates(circ))
    sim = S.Simulator.f64()
    g = F.CircuitGraph.from_circuit(circ)
    st = sim.simulate(g)
    p0 = st.sv.dptr
    assert np.max(np.abs(st.download_amplitudes() - ref)) < 1e-10
    del st
    st2 = sim.simulate(g)
    assert st2.sv.dptr == p0
    assert np.max(np.abs(st2.download_amplitudes() - ref)) < 1e-10
    keep = st2
    st3 = sim.simulate(g)  # the first is still alive: a fresh allocation
    assert st3.sv.dptr != keep.sv.dptr
    del keep, st3
    sim.release_memory()
    assert sim._free == {}
