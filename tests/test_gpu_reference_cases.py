"""The reference's integration-test cases restated against the oracle:

  * tests/cpu_cuda_compare.rs: named gates (H, X, Y, T, Rx, Ry, Rz, CX adjacent,
    non-adjacent and reversed, SWAP, CZ, CCX) and Haar 2q/3q/4q gates on the
    fixed input amp_i ~ (i+1, 0.5 i - 0.25) (:54-69), 1e-10 for FP64 (:27) and
    1e-5 for FP32 (:397);
  * tests/fusion_correctness.rs: populations invariant under fusion widths
    {none, 2, 3, 4} for the QFT with CP + SWAP (:29-42) and the hardware-efficient
    ansatz (:46-64), 1e-10;
  * tests/circuit_execution_order.rs: random 1q/2q Haar circuits with syncs split
    through the sequence (:238-325), 1e-9;
  * tests/density_matrix.rs: depolarizing with p = 0 is the identity (:115-129)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = {1: 1e-10, 0: 1e-5}


@pytest.fixture(scope="module")
def mods(cblib):
    from cast_simulator_b200 import cuda, fusion, simulator, types

    return cuda, fusion, simulator, types


def _run(cu, n, gates, init, prec, sync_every=0):
    spec = cu.CudaKernelGenSpec.f64() if prec == 1 else cu.CudaKernelGenSpec.f32()
    mgr = cu.CudaKernelManager(spec)
    sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
    sv.upload(init)
    for i, g in enumerate(gates):
        mgr.apply(mgr.generate(g), sv)
        if sync_every and (i + 1) % sync_every == 0:
            mgr.sync()
    mgr.sync()
    return sv.download()


def _named(T):
    G = T.QuantumGate
    return [G.h(3), G.x(0), G.y(5), G.t(2), G.rx(0.7, 1), G.ry(-1.3, 4), G.rz(2.1, 6),
            G.cx(2, 3), G.cx(0, 6), G.cx(5, 1), G.swap(1, 6), G.cz(0, 4), G.ccx(0, 3, 5),
            G.s(7), G.cp(0.4, 7, 2)]


@pytest.mark.parametrize("prec", [1, 0])
def test_named_gates_on_fixed_input(mods, oracle, prec):
    cu, F, S, T = mods
    n = 8
    init = oracle.seeded_state(n)
    for g in _named(T):
        ref = init.copy()
        oracle.apply_gate(ref, g.matrix(), g.qubits())
        got = _run(cu, n, [g], init, prec)
        assert np.max(np.abs(got - ref)) < TOL[prec], (g.name, g.qubits())


@pytest.mark.parametrize("prec", [1, 0])
def test_haar_gates_5_to_20_qubits(mods, oracle, prec):
    cu, F, S, T = mods
    rng = np.random.default_rng(138)
    for n in (5, 9, 14, 20):
        init = oracle.seeded_state(n)
        for k in (2, 3, 4):
            q = sorted(int(x) for x in rng.choice(n, size=k, replace=False))
            g = T.QuantumGate.random_unitary(q, rng)
            ref = init.copy()
            oracle.apply_gate(ref, g.matrix(), g.qubits())
            got = _run(cu, n, [g], init, prec)
            assert np.max(np.abs(got - ref)) < TOL[prec], (n, q)


def _hea(T, n, depth):
    c = T.QuantumCircuit(n)
    angle = 0.3
    for d in range(depth):
        for q in range(n):
            c.add(T.QuantumGate.ry(angle, q))
            angle += 0.17
            c.add(T.QuantumGate.rz(angle, q))
            angle += 0.13
        q = d % 2
        while q + 1 < n:
            c.add(T.QuantumGate.cx(q, q + 1))
            q += 2
    return c


@pytest.mark.parametrize("builder", ["qft", "hea"])
def test_fusion_invariance_of_populations(mods, oracle, builder):
    cu, F, S, T = mods
    n = 14
    circ = T.QuantumCircuit.qft(n, True) if builder == "qft" else _hea(T, n, 6)
    ref = np.abs(oracle.simulate(n, [(g.matrix(), g.qubits()) for g in circ.gates()])) ** 2
    for k in (None, 2, 3, 4):
        graph = F.CircuitGraph.from_circuit(circ)
        if k:
            F.optimize(graph, F.FusionConfig.size_only(k))
        pops = S.Simulator.f64().simulate(graph).populations()
        assert np.max(np.abs(pops - ref)) < 1e-10, (builder, k)


def test_execution_order_with_split_syncs(mods, oracle):
    cu, F, S, T = mods
    rng = np.random.default_rng(238)
    n = 14
    gates = []
    for _ in range(100):
        k = int(rng.integers(1, 3))
        q = sorted(int(x) for x in rng.choice(n, size=k, replace=False))
        gates.append(T.QuantumGate.random_unitary(q, rng))
    init = oracle.random_state(n, 5)
    ref = oracle.simulate(n, [(g.matrix(), g.qubits()) for g in gates], init)
    for every in (1, 7, 33):
        got = _run(cu, n, gates, init, 1, sync_every=every)
        assert np.max(np.abs(got - ref)) < 1e-9, every


def test_depolarizing_p0_is_identity_in_dm_mode(mods, oracle):
    cu, F, S, T = mods
    n = 4
    c = T.QuantumCircuit(n)
    for q in range(n):
        c.add(T.QuantumGate.h(q))
    c.add(T.QuantumGate.cx(0, 2))
    c_noisy = T.QuantumCircuit(n)
    for g in c.gates():
        c_noisy.add(g)
    for q in range(n):
        c_noisy.add(T.QuantumGate.depolarizing(q, 0.0))
    a = S.Simulator.f64().simulate(F.CircuitGraph.from_circuit(c), S.Representation.DensityMatrix)
    b = S.Simulator.f64().simulate(F.CircuitGraph.from_circuit(c_noisy), S.Representation.DensityMatrix)
    assert np.max(np.abs(a.populations() - b.populations())) < 1e-12
    assert abs(b.trace() - 1.0) < 1e-12
