"""Gate, noise and circuit types: the host-side mirror of src/types/*.rs.

Mirrors narix10yc/cast_simulator:
  * ``ComplexSquareMatrix`` factories -> numpy complex128 arrays
    (src/types/matrix.rs:51-215);
  * ``QuantumGate`` with canonical ascending qubits (gate.rs:13-45, 483-595),
    ``matmul`` fusion incl. the Cartesian product of Kraus branches
    (gate.rs:280-329), ``to_density_matrix_gate`` (gate.rs:236-257),
    ``scalar_nnz`` / ``arithmetic_intensity`` (gate.rs:261-272) and the noise
    factories (gate.rs:157-227);
  * ``NoiseModel`` (noise.rs:12-33);
  * ``QuantumCircuit`` with ``qft`` and ``eliminate_dead_gates``
    (circuit.rs:117-171), plus the QFT-CX and random-brickwork builders of the
    benchmark configurations.

Convention: gate qubit ``qubits[b]`` is bit ``b`` of the matrix index.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# ── matrix factories (matrix.rs:51-215) ─────────────────────────────────────


def eye(dim: int) -> np.ndarray:
    return np.eye(dim, dtype=np.complex128)


def mat_x():
    return np.array([[0, 1], [1, 0]], dtype=np.complex128)


def mat_y():
    return np.array([[0, -1j], [1j, 0]], dtype=np.complex128)


def mat_z():
    return np.array([[1, 0], [0, -1]], dtype=np.complex128)


def mat_h():
    s = 1.0 / math.sqrt(2.0)
    return np.array([[s, s], [s, -s]], dtype=np.complex128)


def mat_s():
    return np.array([[1, 0], [0, 1j]], dtype=np.complex128)


def mat_t():
    return np.array([[1, 0], [0, complex(math.cos(math.pi / 4), math.sin(math.pi / 4))]],
                    dtype=np.complex128)


def mat_rx(theta):
    c, s = math.cos(theta * 0.5), math.sin(theta * 0.5)
    return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)


def mat_ry(theta):
    c, s = math.cos(theta * 0.5), math.sin(theta * 0.5)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def mat_rz(theta):
    c, s = math.cos(theta * 0.5), math.sin(theta * 0.5)
    return np.array([[complex(c, -s), 0], [0, complex(c, s)]], dtype=np.complex128)


def mat_u3(theta, phi, lam):
    c, s = math.cos(theta * 0.5), math.sin(theta * 0.5)
    eiphi = complex(math.cos(phi), math.sin(phi))
    eilam = complex(math.cos(lam), math.sin(lam))
    eipl = complex(math.cos(phi + lam), math.sin(phi + lam))
    return np.array([[complex(c, 0.0), -eilam * s], [eiphi * s, eipl * c]], dtype=np.complex128)


def mat_cx():
    m = np.zeros((4, 4), dtype=np.complex128)
    m[0, 0] = m[1, 3] = m[2, 2] = m[3, 1] = 1
    return m


def mat_cz():
    return np.diag([1, 1, 1, -1]).astype(np.complex128)


def mat_cp(theta):
    m = eye(4)
    m[3, 3] = complex(math.cos(theta), math.sin(theta))
    return m


def mat_swap():
    m = np.zeros((4, 4), dtype=np.complex128)
    m[0, 0] = m[1, 2] = m[2, 1] = m[3, 3] = 1
    return m


def mat_ccx():
    m = eye(8)
    m[6, 6] = m[7, 7] = 0
    m[6, 7] = m[7, 6] = 1
    return m


def pauli(i: int) -> np.ndarray:
    return [eye(2), mat_x(), mat_y(), mat_z()][i]


# ── helpers (gate.rs:436-680) ────────────────────────────────────────────────


def _canonicalize(matrix: np.ndarray, qubits) -> tuple[np.ndarray, tuple[int, ...]]:
    qubits = [int(q) for q in qubits]
    k = len(qubits)
    if matrix.shape != (1 << k, 1 << k):
        raise ValueError("matrix dimension does not match number of target qubits")
    order = sorted(range(k), key=lambda i: qubits[i])
    sq = [qubits[i] for i in order]
    if any(sq[i] >= sq[i + 1] for i in range(k - 1)):
        raise ValueError("gate qubits must be distinct")
    if order == list(range(k)):
        return matrix, tuple(sq)
    idx = np.arange(1 << k)
    mp = np.zeros(1 << k, dtype=np.int64)
    for p, old in enumerate(order):
        mp |= ((idx >> p) & 1) << old
    return matrix[np.ix_(mp, mp)], tuple(sq)


def _union(a, b) -> tuple[int, ...]:
    return tuple(sorted(set(a) | set(b)))


def expand_matrix(matrix: np.ndarray, gate_qubits, union_qubits) -> np.ndarray:
    """Identity on the union's other wires (gate.rs:436-468)."""
    if tuple(gate_qubits) == tuple(union_qubits):
        return matrix
    pos = [list(union_qubits).index(q) for q in gate_qubits]
    ud = 1 << len(union_qubits)
    tmask = 0
    for p in pos:
        tmask |= 1 << p
    idx = np.arange(ud)
    comp = np.zeros(ud, dtype=np.int64)
    for t, p in enumerate(pos):
        comp |= ((idx >> p) & 1) << t
    rest = idx & ~tmask
    same = rest[:, None] == rest[None, :]
    out = matrix[np.ix_(comp, comp)] * same
    return out.astype(np.complex128)


def superoperator_of(u: np.ndarray) -> np.ndarray:
    """S[r, c] = U[r%d, c%d] * conj(U[r/d, c/d]) (gate.rs:662-680) = kron(conj(U), U)."""
    return np.kron(np.conj(u), u)


# ── noise (noise.rs:12-33) ───────────────────────────────────────────────────


@dataclass
class NoiseModel:
    """Probability-weighted full Kraus operators K_i = V_i · U."""

    branches: list  # [(p, matrix)]

    def __post_init__(self):
        s = 0.0
        for p, _ in self.branches:
            if p < 0:
                raise ValueError(f"noise probability must be non-negative, got {p}")
            s += p
        if abs(s - 1.0) >= 1e-10:
            raise ValueError(f"noise probabilities must sum to 1.0, got {s}")

    def __len__(self):
        return len(self.branches)


# ── QuantumGate (gate.rs:13-329) ─────────────────────────────────────────────


class QuantumGate:
    __slots__ = ("_m", "_q", "_noise", "_name", "_prov", "_op")

    def __init__(self, matrix, qubits, noise: NoiseModel | None = None, name: str = ""):
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))
        self._m, self._q = _canonicalize(m, qubits)
        self._m = np.ascontiguousarray(self._m)
        self._noise = noise
        self._name = name
        self._prov = None
        self._op = None

    def with_provenance(self, index: int) -> "QuantumGate":
        """Copy tagged with a source index; matmul concatenates the tags in
        application order, so a fused gate knows which gates it contains."""
        g = QuantumGate.__new__(QuantumGate)
        g._m, g._q, g._noise, g._name, g._prov = self._m, self._q, self._noise, self._name, [index]
        g._op = self._op
        return g

    def provenance(self):
        return self._prov

    # factories
    @classmethod
    def from_reals(cls, qubits, data):
        d = 1 << len(qubits)
        return cls(np.asarray(data, dtype=np.float64).reshape(d, d).astype(np.complex128), qubits)

    @classmethod
    def _named(cls, mat, qubits, name, params=()):
        """A named standard gate that remembers its OpenQASM form (name, angles,
        operands in the order given), so a circuit of them can be written back."""
        g = cls(mat, qubits, name=name)
        g._op = (name, tuple(float(p) for p in params), tuple(int(q) for q in qubits))
        return g

    @classmethod
    def x(cls, q): return cls._named(mat_x(), [q], "x")
    @classmethod
    def y(cls, q): return cls._named(mat_y(), [q], "y")
    @classmethod
    def z(cls, q): return cls._named(mat_z(), [q], "z")
    @classmethod
    def h(cls, q): return cls._named(mat_h(), [q], "h")
    @classmethod
    def s(cls, q): return cls._named(mat_s(), [q], "s")
    @classmethod
    def t(cls, q): return cls._named(mat_t(), [q], "t")
    @classmethod
    def rx(cls, th, q): return cls._named(mat_rx(th), [q], "rx", (th,))
    @classmethod
    def ry(cls, th, q): return cls._named(mat_ry(th), [q], "ry", (th,))
    @classmethod
    def rz(cls, th, q): return cls._named(mat_rz(th), [q], "rz", (th,))
    @classmethod
    def u3(cls, th, ph, la, q): return cls._named(mat_u3(th, ph, la), [q], "u3", (th, ph, la))
    @classmethod
    def cx(cls, c, t): return cls._named(mat_cx(), [c, t], "cx")
    @classmethod
    def cz(cls, c, t): return cls._named(mat_cz(), [c, t], "cz")
    @classmethod
    def cp(cls, th, c, t): return cls._named(mat_cp(th), [c, t], "cp", (th,))
    @classmethod
    def swap(cls, a, b): return cls._named(mat_swap(), [a, b], "swap")
    @classmethod
    def ccx(cls, a, b, t): return cls._named(mat_ccx(), [a, b, t], "ccx")

    def op(self):
        """(name, angles, operands) of a named standard gate, else None."""
        return self._op

    @classmethod
    def random_unitary(cls, qubits, rng: np.random.Generator):
        """Haar-random unitary by Gram-Schmidt on complex Gaussian rows (matrix.rs:270-308)."""
        qs = sorted(int(q) for q in qubits)
        d = 1 << len(qs)
        m = np.zeros((d, d), dtype=np.complex128)
        for r in range(d):
            while True:
                row = rng.standard_normal(d) + 1j * rng.standard_normal(d)
                for p in range(r):
                    row = row - np.vdot(m[p], row) * m[p]
                nrm = np.linalg.norm(row)
                if nrm > 1e-8:
                    m[r] = row / nrm
                    break
        return cls(m, qs)

    # noise (gate.rs:157-227)
    def with_noise(self, ops) -> "QuantumGate":
        d = self._m.shape[0]
        br = []
        for p, v in ops:
            v = np.asarray(v, dtype=np.complex128)
            if v.shape != (d, d):
                raise ValueError("noise operator dimension must match gate dimension")
            br.append((float(p), v @ self._m))
        g = QuantumGate.__new__(QuantumGate)
        g._m, g._q, g._noise, g._name, g._prov = self._m, self._q, NoiseModel(br), self._name, None
        g._op = None
        return g

    def with_kraus(self, kraus_ops) -> "QuantumGate":
        """Attach a general (non-mixed-unitary) channel sum_i K_i rho K_i^dagger given
        as full Kraus operators of this gate's dimension (K_i already include the gate's
        unitary).  Stored in the reference's weighted form (1/m, sqrt(m) K_i) so that
        S = sum_i p_i K_i (x) conj(K_i) is unchanged (gate.rs:157-171, 246-252)."""
        m = len(kraus_ops)
        br = [(1.0 / m, math.sqrt(m) * np.asarray(k, dtype=np.complex128)) for k in kraus_ops]
        g = QuantumGate.__new__(QuantumGate)
        g._m, g._q, g._noise, g._name, g._prov = self._m, self._q, NoiseModel(br), self._name, None
        g._op = None
        return g

    def with_depolarizing(self, p: float) -> "QuantumGate":
        if self.n_qubits() != 1:
            raise ValueError("depolarizing noise is single-qubit")
        return self.with_noise([(1 - p, eye(2)), (p / 3, mat_x()), (p / 3, mat_y()), (p / 3, mat_z())])

    @classmethod
    def depolarizing(cls, q, p):
        return cls(eye(2), [q]).with_noise(
            [(1 - p, eye(2)), (p / 3, mat_x()), (p / 3, mat_y()), (p / 3, mat_z())])

    @classmethod
    def bit_flip(cls, q, p):
        return cls(eye(2), [q]).with_noise([(1 - p, eye(2)), (p, mat_x())])

    @classmethod
    def phase_flip(cls, q, p):
        return cls(eye(2), [q]).with_noise([(1 - p, eye(2)), (p, mat_z())])

    @classmethod
    def pauli_channel(cls, q, px, py, pz):
        return cls(eye(2), [q]).with_noise(
            [(1 - px - py - pz, eye(2)), (px, mat_x()), (py, mat_y()), (pz, mat_z())])

    @classmethod
    def amplitude_damping(cls, q, gamma):
        """K0 = diag(1, sqrt(1-g)), K1 = sqrt(g)|0><1| (not a reference factory: the
        reference expresses it through with_noise with weights 1/2, see with_kraus)."""
        k0 = np.array([[1, 0], [0, math.sqrt(1 - gamma)]], dtype=np.complex128)
        k1 = np.array([[0, math.sqrt(gamma)], [0, 0]], dtype=np.complex128)
        return cls(eye(2), [q]).with_kraus([k0, k1])

    # accessors
    def matrix(self) -> np.ndarray:
        return self._m

    def qubits(self) -> tuple[int, ...]:
        return self._q

    def n_qubits(self) -> int:
        return len(self._q)

    def effective_n_qubits(self) -> int:
        return self.n_qubits() if self.is_unitary() else 2 * self.n_qubits()

    def is_unitary(self) -> bool:
        return self._noise is None

    def noise_model(self) -> NoiseModel | None:
        return self._noise

    @property
    def name(self) -> str:
        return self._name

    def scalar_nnz(self, ztol: float) -> int:
        m = self._m
        return int(np.count_nonzero(np.abs(m.real) > ztol) + np.count_nonzero(np.abs(m.imag) > ztol))

    def arithmetic_intensity(self, ztol: float) -> float:
        return self.scalar_nnz(ztol) / self._m.shape[0]

    def matmul(self, other: "QuantumGate") -> "QuantumGate":
        """self · other on the union of qubits (other applied first), gate.rs:280-329."""
        uq = _union(self._q, other._q)
        lhs = expand_matrix(self._m, self._q, uq)
        rhs = expand_matrix(other._m, other._q, uq)
        fused = lhs @ rhs
        noise = None
        if self._noise is not None and other._noise is None:
            noise = NoiseModel([(p, expand_matrix(k, self._q, uq) @ rhs) for p, k in self._noise.branches])
        elif self._noise is None and other._noise is not None:
            noise = NoiseModel([(p, lhs @ expand_matrix(k, other._q, uq)) for p, k in other._noise.branches])
        elif self._noise is not None and other._noise is not None:
            br = []
            for pi, ki in self._noise.branches:
                eki = expand_matrix(ki, self._q, uq)
                for qj, kj in other._noise.branches:
                    br.append((pi * qj, eki @ expand_matrix(kj, other._q, uq)))
            noise = NoiseModel(br)
        g = QuantumGate.__new__(QuantumGate)
        g._m, g._q, g._noise, g._name = np.ascontiguousarray(fused), uq, noise, "fused"
        g._prov = (other._prov + self._prov) if (self._prov is not None and other._prov is not None) else None
        g._op = None
        return g

    def to_density_matrix_gate(self, n_total: int) -> "QuantumGate":
        for q in self._q:
            if q >= n_total:
                raise ValueError(f"qubit {q} is out of range for n_total={n_total}")
        if self.is_unitary():
            s = superoperator_of(self._m)
        else:
            d = self._m.shape[0] ** 2
            s = np.zeros((d, d), dtype=np.complex128)
            for p, k in self._noise.branches:
                s += p * superoperator_of(k)
        vq = list(self._q) + [q + n_total for q in self._q]
        return QuantumGate(s, vq)

    def __eq__(self, other):
        return (isinstance(other, QuantumGate) and self._q == other._q
                and np.array_equal(self._m, other._m))

    def __repr__(self):
        return f"QuantumGate({self._name or 'gate'}, qubits={self._q}, noisy={not self.is_unitary()})"


# ── circuits (circuit.rs) ────────────────────────────────────────────────────


class QuantumCircuit:
    def __init__(self, n_qubits: int):
        self._n = int(n_qubits)
        self._gates: list[QuantumGate] = []
        self._measured: list[int] = list(range(self._n))

    def n_qubits(self) -> int:
        return self._n

    def gates(self) -> list[QuantumGate]:
        return self._gates

    def __len__(self):
        return len(self._gates)

    def add(self, gate: QuantumGate) -> "QuantumCircuit":
        for q in gate.qubits():
            if q >= self._n:
                raise ValueError(f"qubit {q} out of range for {self._n}-qubit circuit")
        self._gates.append(gate)
        return self

    def with_measured_qubits(self, qubits) -> "QuantumCircuit":
        for q in qubits:
            if q >= self._n:
                raise ValueError(f"measured qubit {q} out of range for {self._n}-qubit circuit")
        self._measured = list(qubits)
        return self

    def measured_qubits(self):
        return self._measured

    def eliminate_dead_gates(self) -> "QuantumCircuit":
        """Backward liveness from the measured qubits (circuit.rs:117-145)."""
        live = 0
        for q in self._measured:
            live |= 1 << q
        keep = [False] * len(self._gates)
        for i in range(len(self._gates) - 1, -1, -1):
            gm = 0
            for q in self._gates[i].qubits():
                gm |= 1 << q
            if live & gm:
                keep[i] = True
                live |= gm
        out = QuantumCircuit(self._n)
        out._gates = [g for g, k in zip(self._gates, keep) if k]
        out._measured = list(self._measured)
        return out

    @classmethod
    def qft(cls, n: int, swap: bool = True) -> "QuantumCircuit":
        """circuit.rs:151-171: H(i), CP(pi/2^(j-i), j, i) for j > i, then SWAPs."""
        c = cls(n)
        for i in range(n):
            c.add(QuantumGate.h(i))
            for j in range(i + 1, n):
                c.add(QuantumGate.cp(math.pi / float(1 << (j - i)), j, i))
        if swap:
            for i in range(n // 2):
                c.add(QuantumGate.swap(i, n - 1 - i))
        return c

    @classmethod
    def qft_cx(cls, n: int) -> "QuantumCircuit":
        """QFT with CP(t) decomposed as u3(0,0,t/2) c; cx c,t; u3(0,0,-t/2) t; cx c,t;
        u3(0,0,t/2) t - the construction of the reference's tests/assets/qft_14.qasm."""
        c = cls(n)
        for i in range(n):
            c.add(QuantumGate.h(i))
            for j in range(i + 1, n):
                half = math.pi / float(1 << (j - i + 1))
                c.add(QuantumGate.u3(0.0, 0.0, half, i))
                c.add(QuantumGate.cx(i, j))
                c.add(QuantumGate.u3(0.0, 0.0, -half, j))
                c.add(QuantumGate.cx(i, j))
                c.add(QuantumGate.u3(0.0, 0.0, half, j))
        for i in range(n // 2):
            c.add(QuantumGate.swap(i, n - 1 - i))
        return c

    @classmethod
    def brickwork(cls, n: int, depth: int, seed: int, depolarizing: float = 0.0,
                  damping: float = 0.0) -> "QuantumCircuit":
        """Random brickwork: per layer U3 on every qubit (angles uniform in [0, 2pi)
        from a SplitMix64 stream, drawn theta, phi, lambda in qubit order), then CZ on
        (0,1),(2,3),... (even layers) or (1,2),(3,4),... (odd layers).  With noise:
        single-qubit depolarizing(p) on every qubit a gate touches, right after the
        gate, and amplitude damping(gamma) on every qubit at the end of each layer."""
        rng = SplitMix64(seed)
        c = cls(n)
        tau = 2.0 * math.pi
        for layer in range(depth):
            for q in range(n):
                th, ph, la = tau * rng.uniform(), tau * rng.uniform(), tau * rng.uniform()
                c.add(QuantumGate.u3(th, ph, la, q))
                if depolarizing > 0:
                    c.add(QuantumGate.depolarizing(q, depolarizing))
            for q in range(layer & 1, n - 1, 2):
                c.add(QuantumGate.cz(q, q + 1))
                if depolarizing > 0:
                    c.add(QuantumGate.depolarizing(q, depolarizing))
                    c.add(QuantumGate.depolarizing(q + 1, depolarizing))
            if damping > 0:
                for q in range(n):
                    c.add(QuantumGate.amplitude_damping(q, damping))
        return c


class SplitMix64:
    """SplitMix64 (S. Vigna, public domain): the seeded stream behind the circuit
    builders and random states."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.s = seed & self.MASK

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & self.MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / (1 << 53))
