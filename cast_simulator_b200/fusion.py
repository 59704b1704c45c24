"""Circuit graph, gate fusion and cost models.

Host-side mirror of narix10yc/cast_simulator:
  * ``CircuitGraph``: rows x qubits grid with left-push insertion
    (src/circuit_graph.rs:107-504): ``insert_gate`` (303-320),
    ``insert_gate_at_row`` (322-347), ``remove_gate_at`` (349-354),
    ``squeeze`` (356-394), ``fuse_gates_in_same_row`` (403-420),
    ``fuse_gates_across_rows`` (429-461), ``gates_in_row_order`` (490-503);
  * ``optimize``: phase 1 size-2 canonicalisation (src/fusion.rs:14-134) and
    phase 2 agglomerative fusion for cdd_size 3..size_max (fusion.rs:168-345);
  * cost models: ``SizeOnlyCostModel`` (cost_model.rs:20-44),
    ``HardwareAdaptiveCostModel`` (cost_model.rs:238-275) and ``FusionConfig``
    presets (cost_model.rs:286-369), plus ``HardwareProfile`` JSON save/load
    (cost_model.rs:132-226).

The fusion decisions are the reference's; only the container types differ.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field

from .types import QuantumCircuit, QuantumGate

# ── CircuitGraph ─────────────────────────────────────────────────────────────


class CircuitGraph:
    def __init__(self):
        self._n = 0
        self._rows: list[list] = []
        self._gates: list = []  # GateId -> QuantumGate | None

    @classmethod
    def from_circuit(cls, circuit: QuantumCircuit) -> "CircuitGraph":
        g = cls()
        g.ensure_n_qubits(circuit.n_qubits())
        for gate in circuit.gates():
            g.insert_gate(gate)
        return g

    @classmethod
    def from_gates(cls, n_qubits: int, gates) -> "CircuitGraph":
        g = cls()
        g.ensure_n_qubits(n_qubits)
        for gate in gates:
            g.insert_gate(gate)
        return g

    def n_qubits(self) -> int:
        return self._n

    def n_rows(self) -> int:
        return len(self._rows)

    def gate(self, gid):
        return self._gates[gid] if 0 <= gid < len(self._gates) else None

    def gate_id_at(self, row: int, qubit: int):
        if 0 <= row < len(self._rows) and 0 <= qubit < self._n:
            return self._rows[row][qubit]
        return None

    def ensure_n_qubits(self, required: int) -> None:
        if required <= self._n:
            return
        for r in self._rows:
            r.extend([None] * (required - self._n))
        self._n = required

    def _vacant(self, row: int, qubits) -> bool:
        r = self._rows[row]
        return all(q >= len(r) or r[q] is None for q in qubits)

    def _place(self, row: int, gid: int, qubits) -> None:
        r = self._rows[row]
        for q in qubits:
            assert r[q] is None, "row is not vacant for gate placement"
            r[q] = gid

    def insert_gate(self, gate: QuantumGate) -> int:
        qs = gate.qubits()
        self.ensure_n_qubits(max(qs) + 1 if qs else 0)
        min_row = 0
        for q in qs:
            for r in range(len(self._rows) - 1, -1, -1):
                if self._rows[r][q] is not None:
                    min_row = max(min_row, r + 1)
                    break
        row = None
        for r in range(min_row, len(self._rows)):
            if self._vacant(r, qs):
                row = r
                break
        if row is None:
            self._rows.append([None] * self._n)
            row = len(self._rows) - 1
        gid = len(self._gates)
        self._gates.append(gate)
        self._place(row, gid, qs)
        return gid

    def insert_gate_at_row(self, row: int, gate: QuantumGate) -> int:
        assert row < len(self._rows), "row index out of bounds"
        qs = gate.qubits()
        self.ensure_n_qubits(max(qs) + 1 if qs else 0)
        assert self._vacant(row, qs), "target row is not vacant for gate insertion"
        gid = len(self._gates)
        self._gates.append(gate)
        self._place(row, gid, qs)
        return gid

    def remove_gate_at(self, row: int, qubit: int):
        gid = self.gate_id_at(row, qubit)
        if gid is None or self._gates[gid] is None:
            return None
        g = self._gates[gid]
        for q in g.qubits():
            self._rows[row][q] = None
        self._gates[gid] = None
        return g

    def _live_ids_in_row_order(self) -> list[int]:
        out = []
        for r in self._rows:
            seen = []
            for gid in r:
                if gid is not None and gid not in seen:
                    seen.append(gid)
            out.extend(seen)
        return out

    def gates_in_row_order(self) -> list[QuantumGate]:
        return [self._gates[g] for g in self._live_ids_in_row_order()]

    def squeeze(self) -> None:
        ids = self._live_ids_in_row_order()
        rows: list[list] = []
        last = [None] * self._n
        for gid in ids:
            g = self._gates[gid]
            qs = g.qubits()
            mr = max((last[q] + 1 for q in qs if last[q] is not None), default=0)
            row = None
            for r in range(mr, len(rows)):
                if all(rows[r][q] is None for q in qs):
                    row = r
                    break
            if row is None:
                rows.append([None] * self._n)
                row = len(rows) - 1
            for q in qs:
                rows[row][q] = gid
                last[q] = row
        self._rows = rows

    def fuse_gates_in_same_row(self, row: int, qa: int, qb: int):
        a_id, b_id = self.gate_id_at(row, qa), self.gate_id_at(row, qb)
        if a_id is None or b_id is None or a_id == b_id:
            return None
        ga, gb = self._gates[a_id], self._gates[b_id]
        self.remove_gate_at(row, qa)
        self.remove_gate_at(row, qb)
        return self.insert_gate_at_row(row, ga.matmul(gb))

    def fuse_gates_across_rows(self, row_a: int, qa: int, row_b: int, qb: int):
        assert row_b == row_a + 1, "cross-row fusion requires consecutive rows"
        a_id, b_id = self.gate_id_at(row_a, qa), self.gate_id_at(row_b, qb)
        if a_id is None or b_id is None:
            return None
        ga, gb = self._gates[a_id], self._gates[b_id]
        self.remove_gate_at(row_a, qa)
        self.remove_gate_at(row_b, qb)
        fused = gb.matmul(ga)
        if self._vacant(row_b, fused.qubits()):
            target = row_b
        elif self._vacant(row_a, fused.qubits()):
            target = row_a
        else:
            self._rows.insert(row_b, [None] * self._n)
            target = row_b
        return self.insert_gate_at_row(target, fused), target

    def check_consistency(self) -> None:
        seen_rows: dict[int, int] = {}
        for ri, r in enumerate(self._rows):
            assert len(r) == self._n
            for q, gid in enumerate(r):
                if gid is None:
                    continue
                g = self._gates[gid]
                assert g is not None, f"row {ri} references dead gate {gid}"
                assert q in g.qubits()
                assert seen_rows.setdefault(gid, ri) == ri
                for gq in g.qubits():
                    assert r[gq] == gid
        for gid, g in enumerate(self._gates):
            assert (g is not None) == (gid in seen_rows)


# ── cost models (cost_model.rs) ──────────────────────────────────────────────


class SizeOnlyCostModel:
    def __init__(self, max_size: int, max_ai: float = float("inf"), zero_tol: float = 0.0,
                 trajectory_mode: bool = False):
        self.max_size, self.max_ai, self.zero_tol = max_size, max_ai, zero_tol
        self.trajectory_mode = trajectory_mode

    def cost_of(self, gate: QuantumGate) -> float:
        size = gate.n_qubits() if self.trajectory_mode else gate.effective_n_qubits()
        if size > self.max_size:
            return 1.0
        if gate.arithmetic_intensity(self.zero_tol) > self.max_ai:
            return 1.0
        return 1e-10


@dataclass
class HardwareProfile:
    """Roofline profile (cost_model.rs:120-226).  ``tensor_gflops_s`` and
    ``tensor_min_k`` extend the reference's two-segment roofline with the
    tensor-core contraction path: gates with k >= tensor_min_k run there, so
    their compute ceiling is the tensor pipe's (an effective rate that already
    accounts for the 3-pass split precision), not the CUDA cores'."""

    peak_bw_gib_s: float
    peak_gflops_s: float
    bw_slope: float
    crossover_ai: float
    config: dict = field(default_factory=dict)
    raw: list = field(default_factory=list)
    tensor_gflops_s: float = 0.0
    tensor_min_k: int = 0
    # measured register / tile kernel choice per low-target gate class
    # (autotune.tune_kernels records; applied by autotune.apply_kernel_choices)
    kernel_choices: list = field(default_factory=list)

    @staticmethod
    def compute_bw_slope(peak_bw_gib_s: float, scalar_bytes: int) -> float:
        """cost_model.rs:157-159: GFLOP/s per unit AI in the memory-bound regime."""
        return peak_bw_gib_s * (1 << 30) / (2.0 * scalar_bytes) / 1e9

    @classmethod
    def from_roofline(cls, config: dict, peak_bw_gib_s: float, peak_gflops_s: float,
                      scalar_bytes: int) -> "HardwareProfile":
        slope = cls.compute_bw_slope(peak_bw_gib_s, scalar_bytes)
        xo = peak_gflops_s / slope if slope > 0 and peak_gflops_s > 0 else math.inf
        return cls(peak_bw_gib_s, peak_gflops_s, slope, xo, dict(config))

    def crossover_for(self, k: int) -> float:
        if self.tensor_min_k and k >= self.tensor_min_k and self.tensor_gflops_s > 0:
            return self.tensor_gflops_s / self.bw_slope
        return self.crossover_ai

    def save(self, path: str) -> None:
        with open(path, "w") as f:
            json.dump(self.__dict__, f, indent=1)

    @classmethod
    def load(cls, path: str) -> "HardwareProfile":
        with open(path) as f:
            return cls(**json.load(f))


class HardwareAdaptiveCostModel:
    """cost = max(1, AI / crossover) (cost_model.rs:263-275), with the crossover
    taken per gate size from the profile (CUDA-core or tensor-core ceiling)."""

    def __init__(self, profile: HardwareProfile, max_size: int, trajectory_mode: bool = False,
                 zero_tol: float = 0.0):
        self.profile, self.max_size = profile, max_size
        self.trajectory_mode, self.zero_tol = trajectory_mode, zero_tol

    @property
    def crossover_ai(self):
        return self.profile.crossover_ai

    def cost_of(self, gate: QuantumGate) -> float:
        size = gate.n_qubits() if self.trajectory_mode else gate.effective_n_qubits()
        if size > self.max_size:
            return math.inf
        return max(1.0, gate.arithmetic_intensity(self.zero_tol) / self.profile.crossover_for(gate.n_qubits()))


@dataclass
class FusionDecision:
    cdd_size: int
    n_candidates: int
    product_n_qubits: int
    old_cost: float
    new_cost: float
    benefit: float
    accepted: bool


@dataclass
class FusionConfig:
    size_max: int
    benefit_margin: float
    cost_model: object
    trajectory_mode: bool = False
    zero_tol: float = 0.0

    @classmethod
    def size_only(cls, max_size: int = 6) -> "FusionConfig":
        return cls(max_size, 0.0, SizeOnlyCostModel(max_size, zero_tol=0.0), False, 0.0)

    @classmethod
    def size_only_trajectory(cls, max_size: int) -> "FusionConfig":
        return cls(max_size, 0.0, SizeOnlyCostModel(max_size, trajectory_mode=True), True, 0.0)

    @classmethod
    def aggressive(cls) -> "FusionConfig":
        return cls.size_only(6)

    @classmethod
    def default(cls) -> "FusionConfig":
        return cls.size_only(6)

    @classmethod
    def hardware_adaptive(cls, profile: HardwareProfile, max_size: int, zero_tol: float):
        return cls(max_size, 0.0, HardwareAdaptiveCostModel(profile, max_size, False, zero_tol),
                   False, zero_tol)

    @classmethod
    def hardware_adaptive_trajectory(cls, profile: HardwareProfile, max_size: int, zero_tol: float):
        return cls(max_size, 0.0, HardwareAdaptiveCostModel(profile, max_size, True, zero_tol),
                   True, zero_tol)


# ── phase 1: size-2 canonicalisation (fusion.rs:14-134) ──────────────────────


def _absorb_single_qubit_gate(cg: CircuitGraph, row: int, q: int) -> bool:
    gid = cg.gate_id_at(row, q)
    if gid is None:
        return False
    gate = cg.gate(gid)
    if gate is None or gate.n_qubits() != 1:
        return False
    for nr in range(row + 1, cg.n_rows()):
        nid = cg.gate_id_at(nr, q)
        if nid is None:
            continue
        nxt = cg.gate(nid)
        if nxt is None:
            continue
        fused = nxt.matmul(gate)
        cg.remove_gate_at(row, q)
        cg.remove_gate_at(nr, q)
        cg.insert_gate_at_row(nr, fused)
        return True
    for pr in range(row - 1, -1, -1):
        pid = cg.gate_id_at(pr, q)
        if pid is None:
            continue
        prv = cg.gate(pid)
        if prv is None:
            continue
        fused = gate.matmul(prv)
        cg.remove_gate_at(row, q)
        cg.remove_gate_at(pr, q)
        cg.insert_gate_at_row(pr, fused)
        return True
    return False


def _fuse_adjacent_two_qubit_gate(cg: CircuitGraph, row: int, q: int) -> bool:
    lid = cg.gate_id_at(row, q)
    if lid is None:
        return False
    left = cg.gate(lid)
    if left is None or left.n_qubits() != 2 or left.qubits()[0] != q:
        return False
    rid = cg.gate_id_at(row + 1, q)
    if rid is None:
        return False
    right = cg.gate(rid)
    if right is None or right.n_qubits() != 2 or right.qubits() != left.qubits():
        return False
    fused = right.matmul(left)
    cg.remove_gate_at(row, q)
    cg.remove_gate_at(row + 1, q)
    cg.insert_gate_at_row(row + 1, fused)
    return True


def apply_size_two_fusion(cg: CircuitGraph) -> None:
    n = 0
    for row in range(cg.n_rows()):
        for q in range(cg.n_qubits()):
            n += _absorb_single_qubit_gate(cg, row, q)
    if n:
        cg.squeeze()
    n = 0
    row = 0
    while row + 1 < cg.n_rows():
        for q in range(cg.n_qubits()):
            n += _fuse_adjacent_two_qubit_gate(cg, row, q)
        row += 1
    if n:
        cg.squeeze()


# ── phase 2: agglomerative fusion (fusion.rs:168-345) ────────────────────────


def _union_count(a, b) -> int:
    return len(set(a) | set(b))


def _start_fusion(cg: CircuitGraph, config: FusionConfig, cdd: int, start_row: int,
                  start_q: int, log) -> int:
    seed_id = cg.gate_id_at(start_row, start_q)
    if seed_id is None:
        return 0
    seed = cg.gate(seed_id)
    if seed.qubits()[0] != start_q:
        return 0
    tentative = [(seed, start_row)]
    absorbed = {seed_id}
    prod_id, prod_row, prod = seed_id, start_row, seed
    # same-row sweep
    for q in range(start_q + 1, cg.n_qubits()):
        cid = cg.gate_id_at(prod_row, q)
        if cid is None or cid in absorbed:
            continue
        cand = cg.gate(cid)
        if _union_count(prod.qubits(), cand.qubits()) > cdd:
            continue
        tentative.append((cand, prod_row))
        absorbed.add(cid)
        prod_id = cg.fuse_gates_in_same_row(prod_row, prod.qubits()[0], q)
        absorbed.add(prod_id)
        prod = cg.gate(prod_id)
    # cross-row loop
    while True:
        nr = prod_row + 1
        if nr >= cg.n_rows():
            break
        progressed = False
        for q in list(prod.qubits()):
            cid = cg.gate_id_at(nr, q)
            if cid is None or cid in absorbed:
                continue
            cand = cg.gate(cid)
            if _union_count(prod.qubits(), cand.qubits()) > cdd:
                continue
            tentative.append((cand, nr))
            absorbed.add(cid)
            prod_id, prod_row = cg.fuse_gates_across_rows(prod_row, prod.qubits()[0], nr, q)
            absorbed.add(prod_id)
            prod = cg.gate(prod_id)
            progressed = True
            break
        if not progressed:
            break
    if len(tentative) == 1:
        return 0
    old_cost = sum(config.cost_model.cost_of(g) for g, _ in tentative)
    new_cost = config.cost_model.cost_of(prod)
    benefit = old_cost / (new_cost + 1e-10) - 1.0
    accepted = benefit >= config.benefit_margin
    if log is not None:
        log.append(FusionDecision(cdd, len(tentative), prod.effective_n_qubits(), old_cost,
                                  new_cost, benefit, accepted))
    if not accepted:
        cg.remove_gate_at(prod_row, prod.qubits()[0])
        for g, r in tentative:
            cg.insert_gate_at_row(r, g)
        return 0
    return len(tentative) - 1


def apply_gate_fusion(cg: CircuitGraph, config: FusionConfig, cdd: int, log=None) -> int:
    n = 0
    n_rows, n_q = cg.n_rows(), cg.n_qubits()
    for row in range(n_rows):
        for q in range(n_q):
            n += _start_fusion(cg, config, cdd, row, q, log)
    if n:
        cg.squeeze()
    return n


def optimize(cg: CircuitGraph, config: FusionConfig | None = None) -> None:
    config = config or FusionConfig.default()
    apply_size_two_fusion(cg)
    for cdd in range(3, config.size_max + 1):
        while apply_gate_fusion(cg, config, cdd) > 0:
            pass


def optimize_with_log(cg: CircuitGraph, config: FusionConfig) -> list:
    apply_size_two_fusion(cg)
    log: list = []
    for cdd in range(3, config.size_max + 1):
        while apply_gate_fusion(cg, config, cdd, log) > 0:
            pass
    return log


# ── native planner (csrc/fusion.cpp, cast_b200_fuse) ────────────────────────


def _native_config(config: FusionConfig):
    from . import _lib as L

    cm = config.cost_model
    if isinstance(cm, SizeOnlyCostModel):
        if cm.max_ai != float("inf") or cm.trajectory_mode:
            raise ValueError("the native planner supports size-only models without an AI cap")
        return L.FusionConfigC(config.size_max, 0, config.benefit_margin, 0.0, 0.0, 0.0, 0, 0)
    if isinstance(cm, HardwareAdaptiveCostModel):
        p = cm.profile
        txo = p.tensor_gflops_s / p.bw_slope if (p.tensor_min_k and p.tensor_gflops_s > 0) else 0.0
        return L.FusionConfigC(config.size_max, 1, config.benefit_margin, cm.zero_tol,
                               p.crossover_ai, txo, p.tensor_min_k, 0)
    raise ValueError("unsupported cost model for the native planner")


class FusedCircuit:
    """Result of the native planner: fused unitary gates in row order."""

    def __init__(self, handle):
        self.handle = handle

    def __len__(self):
        from . import _lib as L

        return int(L.lib().cast_b200_fused_num_gates(self.handle))

    def gates(self) -> list[QuantumGate]:
        import ctypes as C

        import numpy as np

        from . import _lib as L

        out = []
        k = C.c_uint32()
        q = (C.c_uint32 * 7)()
        for i in range(len(self)):
            L.lib().cast_b200_fused_gate(self.handle, i, C.byref(k), q, None)
            m = np.zeros(1 << (2 * k.value), dtype=np.complex128)
            L.lib().cast_b200_fused_gate(self.handle, i, C.byref(k), q,
                                         m.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)))
            d = 1 << k.value
            out.append(QuantumGate(m.reshape(d, d), [q[j] for j in range(k.value)], name="fused"))
        return out

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                from . import _lib as L

                L.lib().cast_b200_fused_free(h)
            except Exception:
                pass


def optimize_native(n_qubits: int, gates, config: FusionConfig | None = None) -> FusedCircuit:
    """Fuse a unitary gate list (circuit order) with the native planner; same
    decisions as ``optimize`` on ``CircuitGraph.from_gates(n_qubits, gates)``."""
    import ctypes as C

    import numpy as np

    from . import _lib as L

    config = config or FusionConfig.default()
    gates = list(gates)
    for g in gates:
        if not g.is_unitary():
            raise ValueError("the native planner fuses unitary gates only")
    ks = np.array([g.n_qubits() for g in gates], dtype=np.uint32)
    qs = np.array([q for g in gates for q in g.qubits()], dtype=np.uint32)
    ms = (np.concatenate([np.ascontiguousarray(g.matrix()).reshape(-1) for g in gates])
          if gates else np.zeros(1, dtype=np.complex128))
    cfg = _native_config(config)
    eb = L.errbuf()
    h = L.lib().cast_b200_fuse(n_qubits, len(gates), ks.ctypes.data_as(L.c_u32p),
                               qs.ctypes.data_as(L.c_u32p),
                               ms.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)),
                               C.byref(cfg), eb, L.ERR_LEN)
    return FusedCircuit(L.check_ptr(h, eb, "fuse"))
