"""Host-side gate algebra and circuit builders of the product vs the oracle."""

import numpy as np
import pytest

from cast_simulator_b200.types import QuantumCircuit, QuantumGate, SplitMix64


def _as_oracle(circ):
    return [(g.matrix(), g.qubits()) for g in circ.gates()]


def test_builders_match_oracle(oracle):
    for prod, ref in [
        (QuantumCircuit.qft_cx(9), oracle.qft_cx(9)),
        (QuantumCircuit.qft(9, True), oracle.qft_cp(9, True)),
        (QuantumCircuit.brickwork(11, 6, 42), oracle.brickwork(11, 6, 42)),
    ]:
        assert len(prod) == len(ref)
        for g, (m, q) in zip(prod.gates(), ref):
            assert g.qubits() == q
            assert np.max(np.abs(g.matrix() - m)) < 1e-15


def test_splitmix_matches_oracle(oracle):
    import ctypes as C

    st = C.c_uint64(1234)
    r = SplitMix64(1234)
    for _ in range(5):
        assert oracle.lib().or_splitmix64(C.byref(st)) == r.next()


def test_canonicalization_and_errors():
    g = QuantumGate.from_reals([1, 0], [0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0])
    e = QuantumGate.from_reals([0, 1], [0, 0, 1, 0, 0, 0, 0, 1, 1, 0, 0, 0, 0, 1, 0, 0])
    assert g == e
    with pytest.raises(ValueError, match="distinct"):
        QuantumGate(np.eye(4), [0, 0])
    with pytest.raises(ValueError, match="dimension"):
        QuantumGate(np.eye(2), [0, 1])


def test_matmul_matches_oracle(oracle):
    rng = np.random.default_rng(0)
    for _ in range(20):
        qa = sorted(rng.choice(6, size=rng.integers(1, 4), replace=False).tolist())
        qb = sorted(rng.choice(6, size=rng.integers(1, 4), replace=False).tolist())
        a = QuantumGate.random_unitary(qa, rng)
        b = QuantumGate.random_unitary(qb, rng)
        p = a.matmul(b)
        m, q = oracle.matmul((a.matrix(), a.qubits()), (b.matrix(), b.qubits()))
        assert p.qubits() == q and np.max(np.abs(p.matrix() - m)) < 1e-13


def test_noise_fusion_and_dm_lifting(oracle):
    """Cartesian Kraus product under fusion (gate.rs:280-317) and the DM lifting."""
    g = QuantumGate.u3(0.3, 0.2, 0.1, 1).with_depolarizing(0.1)
    h = QuantumGate.cz(0, 1)
    f = h.matmul(g)
    assert len(f.noise_model()) == 4 and f.qubits() == (0, 1)
    n = 3
    dm = f.to_density_matrix_gate(n)
    assert dm.qubits() == (0, 1, 3, 4)
    rho = oracle.dm_zero(n)
    ks = [k for _, k in f.noise_model().branches]
    ws = [p for p, _ in f.noise_model().branches]
    oracle.dm_apply_channel(rho, n, ks, ws, f.qubits())
    rho2 = oracle.dm_zero(n)
    oracle.apply_gate(rho2, dm.matrix(), dm.qubits())
    assert np.max(np.abs(rho - rho2)) < 1e-13


def test_amplitude_damping_channel(oracle):
    g = QuantumGate.amplitude_damping(0, 0.3)
    s = g.to_density_matrix_gate(1)
    rho = np.zeros(4, dtype=complex)
    rho[3] = 1.0  # |1><1|
    oracle.apply_gate(rho, s.matrix(), s.qubits())
    assert abs(rho[0] - 0.3) < 1e-14 and abs(rho[3] - 0.7) < 1e-14


def test_dead_gate_elimination():
    c = QuantumCircuit(3).add(QuantumGate.h(0)).add(QuantumGate.h(2)).add(QuantumGate.cx(0, 1))
    c = c.with_measured_qubits([1])
    assert [g.qubits() for g in c.eliminate_dead_gates().gates()] == [(0,), (0, 1)]


def test_u3_matches_the_openqasm_definition(oracle):
    """Dense U3 (theta != 0, as every brickwork layer uses it) pinned to the
    OpenQASM 2.0 definition, written here from first principles rather than
    from either implementation: U(theta, phi, lambda) =
    e^{i(phi+lambda)/2} Rz(phi) Ry(theta) Rz(lambda), with Rz(a) =
    diag(e^{-ia/2}, e^{ia/2}) and Ry(t) = [[cos t/2, -sin t/2], [sin t/2,
    cos t/2]].  Both the package's and the oracle's U3 must equal it to 1e-15,
    as must the Rx / Ry / Rz of both (U3(t, -pi/2, pi/2) = Rx(t) up to phase is
    the identity the fixtures' decompositions rely on)."""
    rng = np.random.default_rng(9)

    def rz(a):
        return np.diag([np.exp(-0.5j * a), np.exp(0.5j * a)])

    def ry(t):
        c, s = np.cos(t / 2), np.sin(t / 2)
        return np.array([[c, -s], [s, c]], dtype=complex)

    for _ in range(50):
        th, ph, la = rng.uniform(-2 * np.pi, 2 * np.pi, size=3)
        want = np.exp(0.5j * (ph + la)) * rz(ph) @ ry(th) @ rz(la)
        assert np.max(np.abs(QuantumGate.u3(th, ph, la, 0).matrix() - want)) < 1e-15
        assert np.max(np.abs(oracle.named(oracle.U3, th, ph, la) - want)) < 1e-15
        # rotations: Rx(t) = Rz(-pi/2) Ry(t) Rz(pi/2)
        rx = rz(-np.pi / 2) @ ry(th) @ rz(np.pi / 2)
        for mine, ref in ((QuantumGate.rx(th, 0).matrix(), rx), (QuantumGate.ry(th, 0).matrix(), ry(th)),
                          (QuantumGate.rz(th, 0).matrix(), rz(th))):
            assert np.max(np.abs(mine - ref)) < 1e-15
        for kind, ref in ((oracle.RX, rx), (oracle.RY, ry(th)), (oracle.RZ, rz(th))):
            assert np.max(np.abs(oracle.named(kind, th) - ref)) < 1e-15
