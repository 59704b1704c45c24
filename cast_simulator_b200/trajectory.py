"""Batched noisy trajectories: host-side program builder and run API.

Mirror of the reference's ``Simulator::sample_trajectory`` entry point
(src/simulator/trajectory.rs:85-130: ``TrajectoryOpts`` with measured qubits,
sample count and seed; a ``TrajectoryResult`` with a histogram), re-based on
Monte-Carlo quantum-jump trajectories run in one persistent kernel
(``cast_b200_traj_*`` in include/cast_b200.h).

Program construction from a noisy ``QuantumCircuit``:
  * unitary gates between non-Pauli noise operations form a segment that is
    fused with the reference's planner (``fusion.optimize``, size_only(k));
    every gate is tagged with its index, and fused blocks carry the tags of the
    gates they contain in application order;
  * a depolarizing (or bit/phase-flip) channel after gate j on qubit q becomes a
    Pauli error attached to the block containing j, pre-propagated to the end of
    the block: U_j P U_j^dagger with U_j the product of the block's gates after
    j - so errors never split the fusion;
  * consecutive single-qubit amplitude-damping channels with one rate become one
    damping op on a qubit mask; any other single-qubit channel becomes a general
    channel op.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .fusion import CircuitGraph, FusionConfig, optimize
from .types import QuantumCircuit, QuantumGate, eye, expand_matrix, mat_x, mat_y, mat_z

_PAULIS = (mat_x(), mat_y(), mat_z())
_EYE2 = eye(2)


def _close2(a: np.ndarray, b: np.ndarray, tol: float = 1e-9) -> bool:
    """Elementwise |a - b| <= tol for 2x2 matrices, without numpy's per-call
    overhead (the trajectory builder tests every noise site of a circuit)."""
    return all(abs(x - y) <= tol for x, y in zip(a.ravel().tolist(), b.ravel().tolist()))


def _is_pauli_channel(g: QuantumGate):
    """(p, [matrices]) for depolarizing / bit-flip / phase-flip channels on an
    identity base gate, else None."""
    if g.is_unitary() or g.n_qubits() != 1 or not _close2(g.matrix(), _EYE2):
        return None
    br = g.noise_model().branches
    if not _close2(br[0][1], _EYE2):
        return None
    errs = br[1:]
    ps = [p for p, _ in errs]
    mats = [m for _, m in errs]
    for m in mats:
        if not any(_close2(m, P) for P in _PAULIS):
            return None
    if len(errs) == 3 and max(ps) - min(ps) <= 1e-12 * max(1.0, abs(ps[0])):
        return float(sum(ps)), mats
    if len(errs) == 1:
        return float(ps[0]), mats * 3
    return None


def _damping_rate(g: QuantumGate):
    """gamma for an amplitude-damping channel in the weighted-Kraus form
    (weights 1/2, operators sqrt(2) K0, sqrt(2) K1), else None."""
    if g.is_unitary() or g.n_qubits() != 1 or not _close2(g.matrix(), _EYE2):
        return None
    br = g.noise_model().branches
    if len(br) != 2:
        return None
    (p0, a), (p1, b) = br
    k0 = math.sqrt(p0) * a
    k1 = math.sqrt(p1) * b
    if abs(k0[0, 1]) > 1e-12 or abs(k0[1, 0]) > 1e-12 or abs(k0[0, 0] - 1) > 1e-12:
        return None
    gamma = 1.0 - abs(k0[1, 1]) ** 2
    exp1 = np.array([[0, math.sqrt(gamma)], [0, 0]])
    if not _close2(k1, exp1, 1e-12):
        return None
    return gamma


@dataclass
class TrajectoryProgramStats:
    n_blocks: int = 0
    n_errors: int = 0
    n_damping: int = 0
    n_channels: int = 0
    block_sizes: list = field(default_factory=list)  # filled by the Python builder


class TrajectoryProgram:
    """A noisy circuit compiled for the batched-trajectory kernel.  The program
    is built natively (``cast_b200_traj_build``); ``native=False`` runs the
    Python builder, which emits the same program."""

    def __init__(self, circuit: QuantumCircuit, fusion_k: int = 4, native: bool = True):
        if not 1 <= fusion_k <= 4:
            raise ValueError("trajectory fusion width must be 1..4")
        self.n = circuit.n_qubits()
        eb = L.errbuf()
        self.handle = L.check_ptr(L.lib().cast_b200_traj_create(self.n, eb, L.ERR_LEN), eb,
                                  "traj_create")
        self.stats = TrajectoryProgramStats()
        self._k = fusion_k
        if native:
            self._build_native(circuit)
        else:
            self._build(circuit)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().cast_b200_traj_destroy(h)
            except Exception:
                pass

    # -- C ABI helpers
    def _add_gate(self, m, q):
        m = np.ascontiguousarray(m, dtype=np.complex128)
        qq = np.ascontiguousarray(q, dtype=np.uint32)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_traj_add_gate(self.handle, m.view(np.float64).ctypes.data_as(
            C.POINTER(L.Complex64)), qq.ctypes.data_as(L.c_u32p), qq.size, eb, L.ERR_LEN), eb,
            "traj_add_gate")
        self.stats.n_blocks += 1
        self.stats.block_sizes.append(len(q))

    def _add_error(self, p, mats):
        m = np.ascontiguousarray(np.stack(mats), dtype=np.complex128)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_traj_add_pauli_error(self.handle, p, m.view(np.float64).ctypes.data_as(
            C.POINTER(L.Complex64)), eb, L.ERR_LEN), eb, "traj_add_pauli_error")
        self.stats.n_errors += 1

    def _add_damping(self, mask, gamma):
        eb = L.errbuf()
        L.check(L.lib().cast_b200_traj_add_damping(self.handle, mask, gamma, eb, L.ERR_LEN), eb,
                "traj_add_damping")
        self.stats.n_damping += 1

    def _add_channel(self, q, kraus):
        m = np.ascontiguousarray(np.stack(kraus), dtype=np.complex128)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_traj_add_channel(self.handle, q, m.view(np.float64).ctypes.data_as(
            C.POINTER(L.Complex64)), len(kraus), eb, L.ERR_LEN), eb, "traj_add_channel")
        self.stats.n_channels += 1

    # -- construction
    def _flush(self, seg, markers):
        if not seg:
            return
        g = CircuitGraph.from_gates(self.n, seg)
        optimize(g, FusionConfig.size_only(self._k))
        for block in g.gates_in_row_order():
            prov = block.provenance()
            bq = block.qubits()
            self._add_gate(block.matrix(), bq)
            if not any(j in markers for j in prov):
                continue
            # suffix[pos] = product of the block's gates applied after gate pos
            suffix = [None] * len(prov)
            u = eye(1 << len(bq))
            for pos in range(len(prov) - 1, -1, -1):
                suffix[pos] = u
                gi = seg[prov[pos]]
                u = u @ expand_matrix(gi.matrix(), gi.qubits(), bq)
            for pos, j in enumerate(prov):
                for q, p, mats in markers.get(j, ()):
                    u = suffix[pos]
                    ud = u.conj().T
                    prop = [u @ expand_matrix(P, (q,), bq) @ ud for P in mats]
                    self._add_error(p, prop)

    def _build(self, circ: QuantumCircuit):
        seg: list[QuantumGate] = []
        markers: dict[int, list] = {}
        last_on: dict[int, int] = {}
        damp_mask, damp_gamma = 0, None

        def flush_damp():
            nonlocal damp_mask, damp_gamma
            if damp_mask:
                self._add_damping(damp_mask, damp_gamma)
            damp_mask, damp_gamma = 0, None

        for g in circ.gates():
            if g.is_unitary():
                if damp_mask:
                    flush_damp()
                idx = len(seg)
                seg.append(g.with_provenance(idx))
                for q in g.qubits():
                    last_on[q] = idx
                continue
            pc = _is_pauli_channel(g)
            if pc is not None:
                if damp_mask:
                    flush_damp()
                q = g.qubits()[0]
                if q not in last_on:
                    idx = len(seg)
                    seg.append(QuantumGate(eye(2), [q]).with_provenance(idx))
                    last_on[q] = idx
                markers.setdefault(last_on[q], []).append((q, pc[0], pc[1]))
                continue
            # non-Pauli noise closes the unitary segment
            self._flush(seg, markers)
            seg, markers, last_on = [], {}, {}
            gamma = _damping_rate(g)
            q = g.qubits()[0] if g.n_qubits() == 1 else None
            if gamma is not None:
                if damp_mask and (abs(gamma - damp_gamma) > 1e-15 or (damp_mask >> q) & 1):
                    flush_damp()
                damp_mask |= 1 << q
                damp_gamma = gamma
                continue
            if damp_mask:
                flush_damp()
            if g.n_qubits() != 1 or len(g.noise_model()) > 4:
                raise ValueError("trajectory mode supports single-qubit channels with <= 4 Kraus "
                                 "operators")
            kraus = [math.sqrt(p) * k for p, k in g.noise_model().branches]
            self._add_channel(q, kraus)
        self._flush(seg, markers)
        flush_damp()

    def __len__(self):
        return int(L.lib().cast_b200_traj_num_ops(self.handle))

    def _build_native(self, circ: QuantumCircuit) -> None:
        kind, ks, qs, mats, nb, ws = [], [], [], [], [], []
        for g in circ.gates():
            q = g.qubits()
            if g.is_unitary():
                kind.append(0)
                nb.append(0)
            else:
                br = g.noise_model().branches
                if len(q) != 1:
                    raise ValueError("trajectory mode supports single-qubit channels with <= 4 "
                                     "Kraus operators")
                kind.append(1)
                nb.append(len(br))
            ks.append(len(q))
            qs.extend(q)
            mats.append(np.asarray(g.matrix(), dtype=np.complex128).ravel())
            if not g.is_unitary():
                for p, k in br:
                    mats.append(np.asarray(k, dtype=np.complex128).ravel())
                    ws.append(p)
        u32 = lambda a: np.ascontiguousarray(a, dtype=np.uint32)
        kind_a, ks_a, qs_a, nb_a = u32(kind), u32(ks), u32(qs), u32(nb)
        m_a = np.ascontiguousarray(np.concatenate(mats) if mats else np.zeros(1), dtype=np.complex128)
        w_a = np.ascontiguousarray(ws if ws else [0.0], dtype=np.float64)
        stats = np.zeros(4, dtype=np.uint32)
        eb = L.errbuf()
        L.check(L.lib().cast_b200_traj_build(
            self.handle, len(kind), kind_a.ctypes.data_as(L.c_u32p), ks_a.ctypes.data_as(L.c_u32p),
            qs_a.ctypes.data_as(L.c_u32p), m_a.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)),
            nb_a.ctypes.data_as(L.c_u32p), w_a.ctypes.data_as(L.c_dp), self._k,
            stats.ctypes.data_as(L.c_u32p), eb, L.ERR_LEN), eb, "traj_build")
        self.stats.n_blocks, self.stats.n_errors, self.stats.n_damping, self.stats.n_channels = (
            int(x) for x in stats)

    def ops(self) -> list:
        """The program as (kind, k, qubits, probability or rate, mask, matrices)
        tuples, kind one of gate / err / damp / chan (matrices in complex64)."""
        out = []
        names = ("gate", "err", "damp", "chan")
        t, k, m = C.c_uint32(), C.c_uint32(), C.c_uint32()
        nm, p = C.c_uint32(), C.c_double()
        q = np.zeros(4, dtype=np.uint32)
        buf = np.zeros(3 * 256, dtype=np.complex128)
        for i in range(len(self)):
            rc = L.lib().cast_b200_traj_get_op(self.handle, i, C.byref(t), C.byref(k),
                                               q.ctypes.data_as(L.c_u32p), C.byref(p), C.byref(m),
                                               C.byref(nm), buf.view(np.float64).ctypes.data_as(
                                                   C.POINTER(L.Complex64)), buf.size)
            if rc:
                raise RuntimeError("traj_get_op failed")
            kind = names[t.value]
            kk = k.value if kind != "chan" else 1
            d = 1 << kk
            mats = [buf[j * d * d:(j + 1) * d * d].reshape(d, d).copy() for j in range(nm.value)]
            out.append((kind, k.value, tuple(int(x) for x in q[:k.value]), p.value, m.value, mats))
        return out

    def set_launch(self, threads: int = 0, max_ctas: int = 0) -> None:
        """Launch shape of the trajectory kernel: threads per CTA (512 or 1024)
        and the number of CTAs, i.e. trajectories in flight; 0 chooses by the
        number of qubits."""
        eb = L.errbuf()
        L.check(L.lib().cast_b200_traj_set_launch(self.handle, int(threads), int(max_ctas), eb,
                                                  L.ERR_LEN), eb, "traj_set_launch")

    def run(self, n_traj: int, seed: int, stream=None, use_graph: bool = True, first: int = 0):
        """(z, samples): <Z_q> per trajectory (n_traj x n) and one bitstring each,
        for trajectories first .. first + n_traj - 1 of ``seed`` (row j is
        trajectory first + j; a trajectory's draws depend on its index only)."""
        z = np.zeros((n_traj, self.n))
        smp = np.zeros(n_traj, dtype=np.uint32)
        eb = L.errbuf()
        h = stream.handle if stream is not None else None
        L.check(L.lib().cast_b200_traj_run_range(self.handle, first, n_traj, seed & ((1 << 64) - 1),
                                                 z.ctypes.data_as(L.c_dp),
                                                 smp.ctypes.data_as(L.c_u32p), h,
                                                 int(use_graph and h is not None), eb, L.ERR_LEN),
                eb, "traj_run")
        return z, smp


@dataclass
class TrajectoryOpts:
    """trajectory.rs:18-33 (measured qubits, sample count, seed)."""

    measured_qubits: list
    n_samples: int
    seed: int = 0
    fusion_k: int = 4


@dataclass
class TrajectoryResult:
    histogram: dict
    n_samples: int
    z_mean: np.ndarray
    z_stderr: np.ndarray


def sample_trajectory(circuit: QuantumCircuit, opts: TrajectoryOpts, stream=None) -> TrajectoryResult:
    """One Monte-Carlo trajectory per sample; the histogram counts the measured
    qubits' bitstrings (bit j of the key = measured_qubits[j])."""
    prog = TrajectoryProgram(circuit, opts.fusion_k)
    z, smp = prog.run(opts.n_samples, opts.seed, stream)
    hist: dict[int, int] = {}
    for s in smp.tolist():
        key = 0
        for j, q in enumerate(opts.measured_qubits):
            key |= ((s >> q) & 1) << j
        hist[key] = hist.get(key, 0) + 1
    return TrajectoryResult(hist, opts.n_samples, z.mean(axis=0),
                            z.std(axis=0, ddof=1) / math.sqrt(max(1, opts.n_samples)))


def run_plain(circuit: QuantumCircuit, n_traj: int, seed: int, precision=None) -> np.ndarray:
    """Quantum-jump trajectories on the plain per-gate path, one trajectory at a
    time, with every noise decision taken on the host - the execution style of
    the reference's ensemble loop (one launch per gate, a host synchronisation
    at every noisy gate, src/simulator/trajectory.rs:180-265).  Used as the
    baseline that the persistent kernel is measured against.  Returns <Z_q>
    per trajectory (n_traj x n)."""
    from .cuda import CudaPrecision, CudaStatevector
    from .simulator import qubit_populations
    from .types import SplitMix64

    prec = CudaPrecision.F32 if precision is None else precision
    lib = L.lib()
    n = circuit.n_qubits()
    rng = SplitMix64(seed)
    out = np.zeros((n_traj, n))
    tol = 1e-6 if prec == CudaPrecision.F32 else 1e-12

    def apply(sv, m, q):
        mm = np.ascontiguousarray(m, dtype=np.complex128)
        qq = np.ascontiguousarray(q, dtype=np.uint32)
        eb = L.errbuf()
        L.check(lib.cast_b200_apply_gate(sv.dptr, n, int(prec), mm.view(np.float64).ctypes.data_as(
            C.POINTER(L.Complex64)), qq.ctypes.data_as(L.c_u32p), qq.size, tol, tol, None, eb,
            L.ERR_LEN), eb, "apply_gate")

    for t in range(n_traj):
        sv = CudaStatevector(n, prec)
        sv.zero()
        for g in circuit.gates():
            if g.is_unitary():
                apply(sv, g.matrix(), g.qubits())
                continue
            pc = _is_pauli_channel(g)
            if pc is not None:
                u = rng.uniform()
                if u < pc[0]:
                    apply(sv, pc[1][min(2, int(u / pc[0] * 3))], g.qubits())
                continue
            q = g.qubits()[0]
            p1, nrm = qubit_populations(sv)  # host sync at every noisy gate
            kraus = [math.sqrt(p) * k for p, k in g.noise_model().branches]
            probs = []
            for k in kraus:  # ||K psi||^2 from the qubit's populations (K acts on one qubit)
                w0 = abs(k[0, 0]) ** 2 + abs(k[1, 0]) ** 2
                w1 = abs(k[0, 1]) ** 2 + abs(k[1, 1]) ** 2
                cross = 0.0 if abs(np.vdot(k[:, 0], k[:, 1])) < 1e-15 else None
                probs.append(None if cross is None else w0 * (nrm - p1[q]) + w1 * p1[q])
            if any(p is None for p in probs):
                raise ValueError("plain trajectories support channels with orthogonal Kraus columns")
            u = rng.uniform() * sum(probs)
            acc, pick = 0.0, len(kraus) - 1
            for i, p in enumerate(probs):
                acc += p
                if u < acc:
                    pick = i
                    break
            apply(sv, kraus[pick] / math.sqrt(probs[pick] / nrm), g.qubits())
            sv.normalize()
        p1, nrm = qubit_populations(sv)
        out[t] = 1.0 - 2.0 * p1 / nrm
    return out


def run_plain_fused(circuit: QuantumCircuit, n_traj: int, seed: int, precision=None,
                    fusion_k: int = 4, stream=None) -> np.ndarray:
    """Quantum-jump trajectories one at a time on the plain gate kernels, with
    host-side draws: the fair plain-path counterpart of the persistent kernel.

    Each run of unitary gates between two damping layers is fused at width
    ``fusion_k`` once and replayed per trajectory as a CUDA graph (GateProgram).
    Pauli errors (depolarizing) are state-independent, so the host draws them
    per trajectory up front; a segment where one fires runs its gates one by
    one with the Pauli inserted.  A layer of amplitude damping on a qubit mask
    takes one FP64 device reduction (T, D) and one host draw: no jump with
    probability D/T, applied as one renormalised diagonal pass; otherwise the
    jump pattern is sampled qubit by qubit, conditioned on at least one jump
    (populations and masked sums re-read after each step).  Other one-qubit
    channels sample their Kraus branch from the qubit's FP64 populations.
    Returns <Z_q> per trajectory (n_traj x n)."""
    from .cuda import CudaPrecision, CudaStatevector
    from .fusion import optimize_native
    from .simulator import GateProgram, Stream, qubit_populations
    from .types import SplitMix64

    prec = CudaPrecision.F32 if precision is None else precision
    lib = L.lib()
    n = circuit.n_qubits()
    tol = 1e-6 if prec == CudaPrecision.F32 else 1e-12
    st = stream if stream is not None else Stream()
    h = st.handle

    # items: ("seg", gates, sites, program) | ("damp", mask, gamma) | ("chan", gate)
    items: list = []
    seg: list = []
    sites: list = []  # (position after which it acts, qubit, p, [X, Y, Z])

    def close_seg():
        nonlocal seg, sites
        if seg or sites:
            prog = None
            if seg:
                fused = optimize_native(n, seg, FusionConfig.size_only(fusion_k))
                prog = GateProgram(prec, n, tol, tol)
                eb = L.errbuf()
                L.check(lib.cast_b200_program_add_fused(prog.handle, fused.handle, eb, L.ERR_LEN), eb,
                        "program_add_fused")
            items.append(("seg", seg, sites, prog))
        seg, sites = [], []

    for g in circuit.gates():
        if g.is_unitary():
            seg.append(g)
            continue
        pc = _is_pauli_channel(g)
        if pc is not None:
            sites.append((len(seg), g.qubits()[0], pc[0], pc[1]))
            continue
        close_seg()
        gam = _damping_rate(g)
        if gam is not None:
            q = g.qubits()[0]
            last = items[-1] if items else None
            if last is not None and last[0] == "damp" and last[2] == gam and not (last[1] >> q) & 1:
                items[-1] = ("damp", last[1] | (1 << q), gam)
            else:
                items.append(("damp", 1 << q, gam))
        else:
            items.append(("chan", g))
    close_seg()

    def apply(sv, m, q):
        mm = np.ascontiguousarray(m, dtype=np.complex128)
        qq = np.ascontiguousarray(q, dtype=np.uint32)
        eb = L.errbuf()
        L.check(lib.cast_b200_apply_gate(sv.dptr, n, int(prec), mm.view(np.float64).ctypes.data_as(
            C.POINTER(L.Complex64)), qq.ctypes.data_as(L.c_u32p), qq.size, tol, tol, h, eb,
            L.ERR_LEN), eb, "apply_gate")

    def sums(sv, mask, gam):
        t, d = C.c_double(), C.c_double()
        eb = L.errbuf()
        L.check(lib.cast_b200_damping_sums(sv.dptr, n, int(prec), mask, gam, C.byref(t), C.byref(d), h,
                                           eb, L.ERR_LEN), eb, "damping_sums")
        return t.value, d.value

    def scale_popc(sv, mask, factor, scale):
        eb = L.errbuf()
        L.check(lib.cast_b200_scale_popc(sv.dptr, n, int(prec), mask, factor, scale, h, eb, L.ERR_LEN),
                eb, "scale_popc")

    k1_of = lambda gam: np.array([[0, math.sqrt(gam)], [0, 0]], dtype=np.complex128)  # noqa: E731
    rng = SplitMix64(seed)
    out = np.zeros((n_traj, n))
    sv = CudaStatevector(n, prec)
    for t in range(n_traj):
        sv.zero(st)
        for it in items:
            if it[0] == "seg":
                _, gates, ssites, prog = it
                fired = []
                for pos, q, p, mats in ssites:
                    u = rng.uniform()
                    if u < p:
                        fired.append((pos, q, mats[min(2, int(u / p * 3))]))
                if not fired:
                    if prog is not None:
                        prog.run(sv, st, True)
                    continue
                for pos in range(len(gates) + 1):
                    for fp, q, m in fired:
                        if fp == pos:
                            apply(sv, m, (q,))
                    if pos < len(gates):
                        apply(sv, gates[pos].matrix(), gates[pos].qubits())
            elif it[0] == "damp":
                _, mask, gam = it
                tot, w = sums(sv, mask, gam)
                if rng.uniform() * tot < w:  # no jump on any masked qubit
                    scale_popc(sv, mask, math.sqrt(1.0 - gam), 1.0 / math.sqrt(w))
                    continue
                # at least one jump: qubit by qubit, conditioned while none has jumped yet
                rest, jumped = mask, False
                for q in range(n):
                    if not (rest >> q) & 1:
                        continue
                    p1, nrm = qubit_populations(sv, st)
                    pj = gam * p1[q] / nrm
                    if not jumped:
                        tot, w = sums(sv, rest, gam)
                        pj = pj / max(1.0 - w / tot, 1e-300)
                    rest &= ~(1 << q)
                    if rng.uniform() < pj:
                        apply(sv, k1_of(gam) / math.sqrt(gam * p1[q] / nrm), (q,))
                        jumped = True
                    else:
                        scale_popc(sv, 1 << q, math.sqrt(1.0 - gam),
                                   1.0 / math.sqrt(1.0 - gam * p1[q] / nrm))
            else:
                g = it[1]
                q = g.qubits()[0]
                p1, nrm = qubit_populations(sv, st)
                kraus = [math.sqrt(p) * k for p, k in g.noise_model().branches]
                probs = []
                for k in kraus:
                    w0 = abs(k[0, 0]) ** 2 + abs(k[1, 0]) ** 2
                    w1 = abs(k[0, 1]) ** 2 + abs(k[1, 1]) ** 2
                    if abs(np.vdot(k[:, 0], k[:, 1])) >= 1e-15:
                        raise ValueError("plain trajectories support channels with orthogonal Kraus "
                                         "columns")
                    probs.append((w0 * (nrm - p1[q]) + w1 * p1[q]) / nrm)
                u = rng.uniform() * sum(probs)
                acc, pick = 0.0, len(kraus) - 1
                for i, pr in enumerate(probs):
                    acc += pr
                    if u < acc:
                        pick = i
                        break
                apply(sv, kraus[pick] / math.sqrt(probs[pick]), (q,))
        p1, nrm = qubit_populations(sv, st)
        out[t] = 1.0 - 2.0 * p1 / nrm
    return out


def _main(argv=None) -> None:
    """Time one batch of trajectories of the noisy brickwork construction:

        python -m cast_simulator_b200.trajectory --n 16 --depth 30 --traj 4096
    """
    import argparse
    import json
    import time

    from .simulator import Stream

    ap = argparse.ArgumentParser(prog="python -m cast_simulator_b200.trajectory")
    ap.add_argument("--n", type=int, default=16)
    ap.add_argument("--depth", type=int, default=30)
    ap.add_argument("--traj", type=int, default=4096)
    ap.add_argument("--k", type=int, default=3, help="fusion width of the unitary blocks (<= 4)")
    ap.add_argument("--p", type=float, default=1e-3, help="depolarizing after every gate")
    ap.add_argument("--gamma", type=float, default=5e-4, help="amplitude damping per qubit per layer")
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args(argv)
    circ = QuantumCircuit.brickwork(a.n, a.depth, 31337, depolarizing=a.p, damping=a.gamma)
    prog = TrajectoryProgram(circ, a.k)
    st = Stream()
    prog.run(a.traj, 1, st)
    best = float("inf")
    for r in range(a.reps):
        t0 = time.perf_counter()
        prog.run(a.traj, 2 + r, st)
        best = min(best, time.perf_counter() - t0)
    print(json.dumps({"n": a.n, "depth": a.depth, "n_traj": a.traj, "seconds": best,
                      "traj_per_s": a.traj / best, "blocks": prog.stats.n_blocks,
                      "error_sites": prog.stats.n_errors}))


if __name__ == "__main__":
    _main()
