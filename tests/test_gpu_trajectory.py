"""Monte-Carlo trajectories on the GPU vs density-matrix evolution on the CPU
oracle (the reference checks trajectories against its DM simulator at 0.01-0.02,
src/simulator/tests.rs:153-190, 274-316).  Statistical checks use 5 standard
errors of the trajectory mean plus a small floor."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cblib):
    from cast_simulator_b200 import simulator, trajectory, types

    return types, trajectory, simulator


def z_from_pops(pops, n):
    idx = np.arange(pops.size)
    return np.array([1 - 2 * pops[(idx >> q) & 1 == 1].sum() for q in range(n)])


def dm_reference(oracle, circ):
    """Channel-by-channel DM evolution; a unitary gate is merged with the Pauli
    channels that directly follow it so that each superoperator is applied once."""
    n = circ.n_qubits()
    rho = oracle.dm_zero(n)
    gates = circ.gates()
    i = 0
    while i < len(gates):
        g = gates[i]
        if g.is_unitary():
            kraus, weights, qs = [g.matrix()], [1.0], g.qubits()
            j = i + 1
            while j < len(gates) and not gates[j].is_unitary() and set(gates[j].qubits()) <= set(qs) \
                    and len(gates[j].noise_model()) == 4:
                nk, nw = [], []
                pos = qs.index(gates[j].qubits()[0])
                for w0, k0 in zip(weights, kraus):
                    for w1, k1 in gates[j].noise_model().branches:
                        full = _embed(k1, pos, len(qs))
                        nk.append(full @ k0)
                        nw.append(w0 * w1)
                kraus, weights = nk, nw
                j += 1
            oracle.dm_apply_channel(rho, n, kraus, weights, qs)
            i = j
        else:
            br = g.noise_model().branches
            oracle.dm_apply_channel(rho, n, [k for _, k in br], [p for p, _ in br], g.qubits())
            i += 1
    return z_from_pops(oracle.dm_populations(rho, n), n)


def _embed(m1, pos, k):
    out = np.array([[1.0]], dtype=complex)
    for b in range(k - 1, -1, -1):
        out = np.kron(out, m1 if b == pos else np.eye(2))
    return out


def test_noise_free_trajectories_equal_statevector(mods, oracle):
    T, TR, S = mods
    circ = T.QuantumCircuit.brickwork(9, 6, 3)
    sv = oracle.simulate(9, [(g.matrix(), g.qubits()) for g in circ.gates()])
    z_ref = z_from_pops(np.abs(sv) ** 2, 9)
    prog = TR.TrajectoryProgram(circ, 4)
    z, smp = prog.run(64, 1)
    assert np.max(np.abs(z - z_ref[None, :])) < 2e-5
    assert smp.max() < (1 << 9)


@pytest.mark.parametrize("fusion_k", [2, 4])
def test_depolarizing_and_damping_match_dm(mods, oracle, fusion_k):
    T, TR, S = mods
    n = 5
    circ = T.QuantumCircuit.brickwork(n, 4, 17, depolarizing=0.04, damping=0.08)
    z_ref = dm_reference(oracle, circ)
    prog = TR.TrajectoryProgram(circ, fusion_k)
    n_traj = 16384
    st = S.Stream()
    z, _ = prog.run(n_traj, 99, st)
    mean = z.mean(axis=0)
    se = z.std(axis=0, ddof=1) / math.sqrt(n_traj)
    assert np.all(np.abs(mean - z_ref) < 5 * se + 2e-3), (mean, z_ref, se)


def test_strong_damping_rare_path(mods, oracle):
    """Every qubit in |1>, then damping 0.3 on all: the no-jump branch has
    probability 0.7^n, so the exact conditioned sequential path dominates."""
    T, TR, S = mods
    n = 6
    circ = T.QuantumCircuit(n)
    for q in range(n):
        circ.add(T.QuantumGate.x(q))
    for q in range(n):
        circ.add(T.QuantumGate.amplitude_damping(q, 0.3))
    n_traj = 20000
    z, smp = TR.TrajectoryProgram(circ, 2).run(n_traj, 5)
    mean = z.mean(axis=0)
    # each qubit independently decays: P(1) = 0.7 -> <Z> = -0.4
    se = z.std(axis=0, ddof=1) / math.sqrt(n_traj)
    assert np.all(np.abs(mean + 0.4) < 5 * se + 1e-3), mean
    ones = np.array([bin(int(s)).count("1") for s in smp])
    assert abs(ones.mean() - 0.7 * n) < 0.05


def test_general_channel_matches_dm(mods, oracle):
    T, TR, S = mods
    n = 4
    circ = T.QuantumCircuit.brickwork(n, 2, 8)
    # an unequal Pauli channel (not a depolarizing form) -> general channel op
    circ.add(T.QuantumGate.pauli_channel(1, 0.1, 0.05, 0.2))
    circ.add(T.QuantumGate.u3(0.7, 0.1, 0.3, 1))
    z_ref = dm_reference(oracle, circ)
    prog = TR.TrajectoryProgram(circ, 3)
    assert prog.stats.n_channels == 1
    n_traj = 20000
    z, _ = prog.run(n_traj, 3)
    se = z.std(axis=0, ddof=1) / math.sqrt(n_traj)
    assert np.all(np.abs(z.mean(axis=0) - z_ref) < 5 * se + 1e-3)


@pytest.mark.timeout(600)
def test_trajectory_config_10q_instance_vs_dm(mods, oracle):
    """The trajectory configuration's construction (brickwork depth 30, depolarizing
    1e-3 after every gate, damping 5e-4 per qubit per layer) at 10 qubits, 4096
    trajectories vs the DM oracle."""
    T, TR, S = mods
    n = 10
    circ = T.QuantumCircuit.brickwork(n, 30, 2024, depolarizing=1e-3, damping=5e-4)
    z_ref = dm_reference(oracle, circ)
    z, _ = TR.TrajectoryProgram(circ, 4).run(4096, 7, S.Stream())
    mean = z.mean(axis=0)
    se = z.std(axis=0, ddof=1) / math.sqrt(4096)
    assert np.all(np.abs(mean - z_ref) < 5 * se + 2e-3), (np.abs(mean - z_ref).max(), se.max())


def test_graph_replay_is_deterministic(mods):
    T, TR, S = mods
    circ = T.QuantumCircuit.brickwork(8, 5, 1, depolarizing=0.02, damping=0.02)
    prog = TR.TrajectoryProgram(circ, 4)
    st = S.Stream()
    a, sa = prog.run(300, 11, st)
    b, sb = prog.run(300, 11, st)
    c, _ = prog.run(300, 12, st)
    assert np.array_equal(a, b) and np.array_equal(sa, sb)
    assert not np.array_equal(a, c)


# State sizes from well inside L2 (12 qubits: 32 KB a trajectory) to beyond it
# (18 qubits: 2 MB a trajectory, 296 MB for 148 at once), with gates on the
# lowest and highest qubits; both CTA sizes of the kernel.
LAYOUT_NS = [12, 14, 15, 16, 17, 18]


@pytest.mark.parametrize("threads", [512, 1024])
@pytest.mark.parametrize("n", LAYOUT_NS)
def test_layouts_noise_free_equal_statevector(mods, oracle, n, threads):
    T, TR, S = mods
    circ = T.QuantumCircuit.brickwork(n, 6, 40 + n)
    sv = oracle.simulate(n, [(g.matrix(), g.qubits()) for g in circ.gates()])
    z_ref = z_from_pops(np.abs(sv) ** 2, n)
    n_traj = 2048
    prog = TR.TrajectoryProgram(circ, 4)
    prog.set_launch(threads)
    z, smp = prog.run(n_traj, 21, S.Stream())
    assert np.max(np.abs(z - z_ref[None, :])) < 2e-5
    assert smp.max() < (1 << n)
    # sampled bitstrings: P(bit q = 1) = (1 - <Z_q>) / 2
    bits = (smp[:, None].astype(np.int64) >> np.arange(n)[None, :]) & 1
    p1 = (1 - z_ref) / 2
    se = np.sqrt(np.maximum(p1 * (1 - p1), 1e-4) / n_traj)
    assert np.all(np.abs(bits.mean(axis=0) - p1) < 5 * se + 1e-3)


def _spread(circ, T, n, active):
    """The circuit's gates on qubits active[0] < active[1] < ... of an n-qubit
    register (an order-preserving relabelling keeps every matrix as it is)."""
    out = T.QuantumCircuit(n)
    for g in circ.gates():
        out.add(T.QuantumGate(g.matrix(), [active[q] for q in g.qubits()], g.noise_model()))
    return out


@pytest.mark.parametrize("n", LAYOUT_NS)
def test_layouts_noisy_embedded_match_dm(mods, oracle, n):
    """A noisy 6-qubit brickwork (depolarizing, damping, an unequal Pauli
    channel) placed on low, boundary and top qubits of an n-qubit register:
    the active qubits follow the 6-qubit DM oracle, idle qubits stay in |0>."""
    T, TR, S = mods
    small = T.QuantumCircuit.brickwork(6, 4, 77, depolarizing=0.03, damping=0.06)
    small.add(T.QuantumGate.pauli_channel(5, 0.1, 0.05, 0.2))
    small.add(T.QuantumGate.u3(0.7, 0.1, 0.3, 5))
    z_ref = dm_reference(oracle, small)
    active = [0, n // 3, n - 4, n - 3, n - 2, n - 1]
    prog = TR.TrajectoryProgram(_spread(small, T, n, active), 3)
    assert prog.stats.n_channels == 1
    n_traj = 8192
    z, smp = prog.run(n_traj, 1234 + n, S.Stream())
    mean = z.mean(axis=0)
    se = z.std(axis=0, ddof=1) / math.sqrt(n_traj)
    assert np.all(np.abs(mean[active] - z_ref) < 5 * se[active] + 2e-3), (mean[active], z_ref)
    idle = [q for q in range(n) if q not in active]
    assert np.max(np.abs(z[:, idle] - 1.0)) < 1e-5
    assert np.all((smp.astype(np.int64) >> np.array(idle)[:, None] & 1) == 0)


@pytest.mark.parametrize("n", [14, 16])
def test_replay_is_deterministic_both_cta_sizes(mods, n):
    T, TR, S = mods
    circ = T.QuantumCircuit.brickwork(n, 3, 5, depolarizing=0.02, damping=0.02)
    prog = TR.TrajectoryProgram(circ, 3)
    st = S.Stream()
    a, sa = prog.run(600, 11, st)
    b, sb = prog.run(600, 11, st)
    assert np.array_equal(a, b) and np.array_equal(sa, sb)


def test_trajectories_leave_gate_throughput_alone(mods):
    """A trajectory run must leave no context-wide state behind that slows the
    statevector passes that follow in the same process (a persisting-L2
    set-aside once cut them to less than half)."""
    from cast_simulator_b200 import cuda as cu
    from cast_simulator_b200.fusion import FusionConfig, optimize_native

    T, TR, S = mods
    n = 26
    gates = optimize_native(n, T.QuantumCircuit.brickwork(n, 8, 3).gates(), FusionConfig.size_only(4)).gates()
    prog = S.GateProgram(cu.CudaPrecision.F64, n, 1e-12, 1e-12, False)
    for g in gates:
        prog.add(g.matrix(), g.qubits())
    sv = cu.CudaStatevector(n, cu.CudaPrecision.F64)
    st = S.Stream()

    def best_time():
        e0, e1, ts = S.Event(), S.Event(), []
        for _ in range(4):
            sv.zero(st)
            e0.record(st)
            prog.run(sv, st, use_graph=True)
            e1.record(st)
            e1.sync()
            ts.append(e1.elapsed_s(e0))
        return min(ts)

    before = best_time()
    TR.TrajectoryProgram(T.QuantumCircuit.brickwork(16, 10, 1, depolarizing=1e-3, damping=5e-4), 3).run(
        1024, 1, st)
    after = best_time()
    # the slowdown this guards against was 2x or more; the margin leaves room
    # for SM clock changes under the power cap between the two measurements
    assert after < 1.5 * before, (before, after)


@pytest.mark.parametrize("n", [12, 16])
def test_ranges_reproduce_the_batch(mods, n):
    """Trajectory i draws from Philox stream (seed, i) whatever range it runs
    in: two ranges reproduce one batch row for row, which is what the
    data-parallel runner relies on."""
    from cast_simulator_b200 import distributed as D

    T, TR, S = mods
    circ = T.QuantumCircuit.brickwork(n, 4, 9, depolarizing=0.02, damping=0.02)
    prog = TR.TrajectoryProgram(circ, 3)
    st = S.Stream()
    z, smp = prog.run(300, 5, st)
    z1, s1 = prog.run(100, 5, st, first=0)
    z2, s2 = prog.run(200, 5, st, first=100)
    assert np.array_equal(np.concatenate([z1, z2]), z)
    assert np.array_equal(np.concatenate([s1, s2]), smp)
    mean, rows, first = D.run_trajectories_sharded(prog, 300, 5, st)
    assert first == 0 and np.array_equal(rows, z)
    assert np.allclose(mean, z.mean(axis=0), atol=1e-14)


def test_plain_fused_trajectories_match_dm(mods, oracle):
    """The host-driven plain-path trajectories (fused graph segments, host
    Pauli draws, one masked FP64 reduction per damping layer) against the DM
    oracle: strong noise so that every branch kind is taken."""
    T, TR, S = mods
    n = 5
    circ = T.QuantumCircuit.brickwork(n, 4, 17, depolarizing=0.04, damping=0.08)
    z_ref = dm_reference(oracle, circ)
    n_traj = 3000
    z = TR.run_plain_fused(circ, n_traj, 11, fusion_k=3)
    se = z.std(axis=0, ddof=1) / math.sqrt(n_traj)
    assert np.all(np.abs(z.mean(axis=0) - z_ref) < 5 * se + 2e-3), (z.mean(axis=0), z_ref, se)


def test_plain_fused_conditioned_jump_path(mods):
    """Every qubit in |1>, damping 0.3 on all: the no-jump branch has
    probability 0.7^n, so the conditioned qubit-by-qubit path dominates;
    each qubit decays independently, <Z> = -0.4."""
    T, TR, S = mods
    n = 6
    circ = T.QuantumCircuit(n)
    for q in range(n):
        circ.add(T.QuantumGate.x(q))
    for q in range(n):
        circ.add(T.QuantumGate.amplitude_damping(q, 0.3))
    n_traj = 3000
    z = TR.run_plain_fused(circ, n_traj, 5, fusion_k=2)
    se = z.std(axis=0, ddof=1) / math.sqrt(n_traj)
    assert np.all(np.abs(z.mean(axis=0) + 0.4) < 5 * se + 1e-3), z.mean(axis=0)


def test_plain_fused_general_channel(mods, oracle):
    T, TR, S = mods
    n = 4
    circ = T.QuantumCircuit.brickwork(n, 2, 8)
    circ.add(T.QuantumGate.pauli_channel(1, 0.1, 0.05, 0.2))
    circ.add(T.QuantumGate.u3(0.7, 0.1, 0.3, 1))
    z_ref = dm_reference(oracle, circ)
    n_traj = 3000
    z = TR.run_plain_fused(circ, n_traj, 3, fusion_k=3)
    se = z.std(axis=0, ddof=1) / math.sqrt(n_traj)
    assert np.all(np.abs(z.mean(axis=0) - z_ref) < 5 * se + 1e-3)


@pytest.mark.parametrize("prec", [1, 0])
def test_damping_sums_and_popcount_scale(mods, oracle, prec):
    """cast_b200_damping_sums / cast_b200_scale_popc against numpy on a random
    state: FP64 sums (1e-12 relative for complex128, 1e-6 for complex64) and the
    masked diagonal pass."""
    import ctypes as C

    from cast_simulator_b200 import _lib as L
    from cast_simulator_b200 import cuda as cu

    n, mask, gam = 13, 0b1010010110011, 0.23
    psi = oracle.random_state(n, 4)
    sv = cu.CudaStatevector(n, cu.CudaPrecision(prec))
    sv.upload(psi)
    psi = sv.download()  # the values the device holds (complex64-rounded for prec 0)
    idx = np.arange(1 << n)
    pc = np.array([bin(int(i & mask)).count("1") for i in idx])
    p = np.abs(psi) ** 2
    t, d = C.c_double(), C.c_double()
    eb = L.errbuf()
    lib = L.lib()
    L.check(lib.cast_b200_damping_sums(sv.dptr, n, prec, mask, gam, C.byref(t), C.byref(d), None, eb,
                                       L.ERR_LEN), eb, "damping_sums")
    rel = 1e-12 if prec == 1 else 1e-6
    assert abs(t.value - p.sum()) <= rel * p.sum()
    assert abs(d.value - (p * (1 - gam) ** pc).sum()) <= rel * p.sum()
    f, sc = math.sqrt(1 - gam), 1.0 / math.sqrt(d.value)
    L.check(lib.cast_b200_scale_popc(sv.dptr, n, prec, mask, f, sc, None, eb, L.ERR_LEN), eb,
            "scale_popc")
    got = sv.download()
    want = psi * sc * f ** pc
    assert np.max(np.abs(got - want)) < (1e-14 if prec == 1 else 1e-6)
    assert abs(np.sum(np.abs(got) ** 2) - 1.0) < (1e-12 if prec == 1 else 1e-5)
