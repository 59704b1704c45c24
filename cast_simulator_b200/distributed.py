"""Statevector sharded over G = 2^g ranks (one process per GPU) with qubit-swap
exchanges.

The reference runs one statevector on one device; this is the multi-GPU form of
the same gate-application path:

  * **Layout.** There are n logical qubits and L = n - g local physical
    positions per rank. Rank r holds the 2^L amplitudes whose top g physical
    qubits equal the bits of r. ``perm[logical] = physical`` records which
    logical qubit currently sits at which physical position; it starts as the
    identity.
  * **Local gates.** A gate whose physical targets are all below L runs on every
    rank's shard locally, through the device kernel (C ABI) on GPU ranks.
  * **Global targets.** Before a gate touches a global position P = L + b, that
    position is swapped with a local position p the gate does not use. Rank r
    and its partner r ^ 2^b exchange the half of their shards whose local bit p
    differs from their own bit b: 2^(L-1) amplitudes, with no collective, sent
    in chunks through two fixed staging buffers (``chunk_amps`` amplitudes each,
    allocated once), so an exchange needs no half-shard temporaries and the
    shard can fill most of the device. The two positions then trade logical
    qubits in ``perm``.
  * **Which local position.** ``apply`` takes the highest free one.
    ``apply_circuit`` looks ahead: it evicts the local position whose logical
    qubit is next used furthest in the future (never, if possible) - Belady's
    rule, which minimises the number of exchanges over the circuit.
  * **Reading out.** ``gather`` assembles the logical-order state on rank 0.
    ``expectation_z`` all-reduces per-position populations (FP64) and maps them
    back to logical qubits.

Trajectories shard without any exchange: ``run_trajectories_sharded`` gives
rank r a contiguous range of trajectory indices (each trajectory's draws depend
on its index only, so the union of the ranges is the single-GPU batch row for
row) and all-reduces the per-qubit <Z> sums in FP64.

Communication is ``torch.distributed``: NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np

LocalApply = Callable[[object, np.ndarray, tuple], None]


def swap_plan(targets_phys: tuple, n_local: int, in_use: set | None = None,
              priority: Callable[[int], float] | None = None) -> list[tuple[int, int]]:
    """(global position, local position) swaps that make every physical target
    local.

    Each global target is paired with a local position that is neither a target
    of this gate nor already chosen: the one with the largest ``priority``
    (ties, and no priority, go to the highest position)."""
    in_use = set(in_use or ()) | {q for q in targets_phys if q < n_local}
    plan = []
    for q in sorted(q for q in targets_phys if q >= n_local):
        free = [c for c in range(n_local - 1, -1, -1) if c not in in_use]
        if not free:
            raise ValueError("gate is wider than the local qubits of a shard")
        p = max(free, key=priority) if priority else free[0]
        in_use.add(p)
        plan.append((q, p))
    return plan


def next_uses(gates_qubits: list[tuple], n_qubits: int) -> list[dict]:
    """For every gate index i, {logical qubit: index of its next use after i}
    for the qubits used again later (others are absent: never used again)."""
    out: list[dict] = [dict() for _ in gates_qubits]
    upcoming: dict = {}
    for i in range(len(gates_qubits) - 1, -1, -1):
        out[i] = dict(upcoming)
        for q in gates_qubits[i]:
            upcoming[q] = i
    return out


def permute_bits(index: np.ndarray, perm: list[int]) -> np.ndarray:
    """Physical index of every logical index: bit perm[i] of the result is bit i
    of ``index``."""
    out = np.zeros_like(index)
    for logical, physical in enumerate(perm):
        out |= ((index >> logical) & 1) << physical
    return out


class ShardedStatevector:
    """One rank's shard of a 2^n statevector.

    ``shard`` is a 1-D complex tensor of 2^(n-g) amplitudes (torch; CUDA on GPU
    ranks, CPU with gloo). ``apply_local(shard, matrix, local_qubits)`` applies
    a gate to the shard in place. On GPU ranks, ``cuda_apply_local`` runs the
    device kernels through the C ABI."""

    def __init__(self, n_qubits: int, shard, apply_local: LocalApply, group=None,
                 chunk_amps: int = 1 << 24):
        """chunk_amps: amplitudes an exchange moves per send/recv (a power of
        two; two staging buffers of this size are allocated on the shard's
        device the first time an exchange runs)."""
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        g = int(round(math.log2(self.world)))
        if 1 << g != self.world:
            raise ValueError("the number of ranks must be a power of two")
        self.n, self.g, self.n_local = int(n_qubits), g, int(n_qubits) - g
        if self.n_local < 1 or shard.numel() != (1 << self.n_local):
            raise ValueError("shard must hold 2^(n - log2(world)) amplitudes")
        if chunk_amps < 1 or chunk_amps & (chunk_amps - 1):
            raise ValueError("chunk_amps must be a power of two")
        self.shard = shard
        self.apply_local = apply_local
        self.perm = list(range(self.n))  # logical -> physical position
        self.n_exchanges = 0
        self.exchanged_amps = 0
        self.chunk_amps = min(int(chunk_amps), max(1, 1 << (self.n_local - 1)))
        self._stage = None  # (send, recv) staging buffers

    # -- state ------------------------------------------------------------------
    def set_zero(self) -> None:
        self.shard.zero_()
        if self.rank == 0:
            self.shard[0] = 1.0
        self.perm = list(range(self.n))

    # -- gates ------------------------------------------------------------------
    def apply(self, matrix: np.ndarray, qubits) -> None:
        """Apply a gate given on logical qubits (in the order of the matrix's
        index bits)."""
        self._apply(matrix, qubits, None)

    def apply_circuit(self, gates) -> None:
        """Apply gates (objects with ``matrix()`` and ``qubits()``, logical
        qubits) in order, choosing the local position each exchange evicts by
        look-ahead over the rest of the list."""
        gates = list(gates)
        nxt = next_uses([tuple(g.qubits()) for g in gates], self.n)
        for i, g in enumerate(gates):
            self._apply(g.matrix(), g.qubits(), nxt[i])

    def _apply(self, matrix, qubits, next_use: dict | None) -> None:
        phys = tuple(self.perm[q] for q in qubits)
        prio = None
        if next_use is not None:
            at = {p: lq for lq, p in enumerate(self.perm)}  # physical -> logical
            prio = lambda pos: next_use.get(at[pos], math.inf)  # noqa: E731
        for gpos, lpos in swap_plan(phys, self.n_local, priority=prio):
            self._swap(gpos, lpos)
        phys = tuple(self.perm[q] for q in qubits)
        self.apply_local(self.shard, np.ascontiguousarray(matrix), phys)

    def _blocks(self, lpos: int, half: int):
        """The half of the shard whose local bit lpos is `half`, as views of at
        most chunk_amps amplitudes each, in the order both partners walk them:
        the shard is (rows, 2, run) with run = 2^lpos; a block is a slice of one
        run, or whole runs of consecutive rows (a strided view)."""
        run = 1 << lpos
        rows = 1 << (self.n_local - lpos - 1)
        c = self.chunk_amps
        view = self.shard.view(rows, 2, run)
        if run >= c:
            for r in range(rows):
                for off in range(0, run, c):
                    yield view[r, half, off:off + c]
        else:
            per = c // run
            for r0 in range(0, rows, per):
                yield view[r0:r0 + per, half, :]

    def _swap(self, gpos: int, lpos: int) -> None:
        """Exchange global position gpos with local position lpos."""
        import torch

        b = gpos - self.n_local
        my_bit = (self.rank >> b) & 1
        partner = self.rank ^ (1 << b)
        if self._stage is None:
            self._stage = (torch.empty(self.chunk_amps, dtype=self.shard.dtype, device=self.shard.device),
                           torch.empty(self.chunk_amps, dtype=self.shard.dtype, device=self.shard.device))
        send, recv = self._stage
        for blk in self._blocks(lpos, 1 - my_bit):
            cnt = blk.numel()
            send[:cnt].view(blk.shape).copy_(blk)
            # real views: not every backend transfers complex tensors
            ops = [self.dist.P2POp(self.dist.isend, torch.view_as_real(send[:cnt]), partner, self.group),
                   self.dist.P2POp(self.dist.irecv, torch.view_as_real(recv[:cnt]), partner, self.group)]
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
            blk.copy_(recv[:cnt].view(blk.shape))
            self.exchanged_amps += cnt
        la = self.perm.index(gpos)
        lb = self.perm.index(lpos)
        self.perm[la], self.perm[lb] = lpos, gpos
        self.n_exchanges += 1

    # -- read-out -----------------------------------------------------------------
    def gather(self) -> np.ndarray | None:
        """The full statevector in logical qubit order on rank 0 (None
        elsewhere)."""
        import torch

        parts = [torch.empty_like(self.shard) for _ in range(self.world)] if self.rank == 0 else None
        if self.world == 1:
            parts = [self.shard]
        else:
            self.dist.gather(torch.view_as_real(self.shard),
                             [torch.view_as_real(x) for x in parts] if parts else None,
                             dst=0, group=self.group)
        if self.rank != 0:
            return None
        phys = np.concatenate([p.cpu().numpy() for p in parts])
        idx = np.arange(1 << self.n, dtype=np.int64)
        return phys[permute_bits(idx, self.perm)]

    def expectation_z(self) -> np.ndarray:
        """<Z_q> for every logical qubit, every rank (FP64 all-reduce)."""
        import torch

        if self.shard.is_cuda:
            # one FP64 device pass over the shard for every local qubit
            # (cast_b200_qubit_populations), on torch's current stream
            import ctypes as C

            from . import _lib as L

            pop = np.zeros(max(1, self.n_local), dtype=np.float64)
            nrm = C.c_double()
            eb = L.errbuf()
            stream = torch.cuda.current_stream(self.shard.device).cuda_stream
            prec = 1 if self.shard.dtype == torch.complex128 else 0
            L.check(L.lib().cast_b200_qubit_populations(
                self.shard.data_ptr(), self.n_local, prec, pop.ctypes.data_as(L.c_dp), C.byref(nrm),
                C.c_void_p(stream) if stream else None, eb, L.ERR_LEN), eb, "qubit_populations")
            host = np.zeros(self.n + 1, dtype=np.float64)
            host[:self.n_local] = pop[:self.n_local]
            tot = nrm.value
            ones = torch.tensor(host, dtype=torch.float64, device=self.shard.device)
        else:
            p = torch.view_as_real(self.shard).to(torch.float64).square().sum(-1)  # |psi|^2 in FP64
            ones = torch.zeros(self.n + 1, dtype=torch.float64, device=p.device)
            idx = torch.arange(1 << self.n_local, device=p.device)
            for pos in range(self.n_local):
                ones[pos] = p[((idx >> pos) & 1) == 1].sum()
            tot = p.sum()
        for b in range(self.g):
            ones[self.n_local + b] = tot if (self.rank >> b) & 1 else 0.0
        ones[self.n] = tot
        if self.world > 1:
            self.dist.all_reduce(ones, group=self.group)
        ones = ones.cpu().numpy()
        return np.array([1.0 - 2.0 * ones[self.perm[q]] / ones[self.n] for q in range(self.n)])


def cuda_apply_local(precision: int, ztol: float = 1e-12, otol: float = 1e-12) -> LocalApply:
    """Local applier for GPU ranks: the device gate kernels through
    ``cast_b200_apply_gate`` on the shard's memory, ordered on torch's current
    stream."""
    import ctypes as C

    import torch

    from . import _lib as L

    from .types import _canonicalize

    def apply(shard, matrix, phys_qubits):
        # the kernels take ascending qubits: permute the matrix's index bits
        m, srt = _canonicalize(np.asarray(matrix, dtype=np.complex128), list(phys_qubits))
        qs = np.asarray(srt, dtype=np.uint32)
        k = len(srt)
        m = np.ascontiguousarray(m)
        n_local = int(round(math.log2(shard.numel())))
        eb = L.errbuf()
        stream = torch.cuda.current_stream(shard.device).cuda_stream
        L.check(L.lib().cast_b200_apply_gate(
            shard.data_ptr(), n_local, precision, m.view(np.float64).ctypes.data_as(C.POINTER(L.Complex64)),
            qs.ctypes.data_as(L.c_u32p), k, ztol, otol, C.c_void_p(stream), eb, L.ERR_LEN), eb, "apply_gate")

    return apply


def trajectory_range(n_traj: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of rank's contiguous share of n_traj trajectories; the
    first n_traj % world ranks take one more."""
    if world < 1 or not 0 <= rank < world or n_traj < 0:
        raise ValueError("bad trajectory partition")
    base, rem = divmod(n_traj, world)
    return rank * base + min(rank, rem), base + (1 if rank < rem else 0)


def run_trajectories_sharded(program, n_traj: int, seed: int, stream=None, group=None):
    """Data-parallel trajectories over the ranks of ``group``: each rank runs its
    range of ``program`` (a ``TrajectoryProgram``) and the per-qubit sums of
    <Z> plus the trajectory count are all-reduced in FP64.  Returns
    (mean <Z> over all n_traj trajectories, this rank's rows, this rank's first
    index)."""
    import torch
    import torch.distributed as dist

    on = dist.is_initialized()
    world = dist.get_world_size(group) if on else 1
    rank = dist.get_rank(group) if on else 0
    first, count = trajectory_range(n_traj, world, rank)
    n = program.n
    if count:
        z, _ = program.run(count, seed, stream, first=first)
    else:
        z = np.zeros((0, n))
    dev = "cuda" if on and dist.get_backend(group) == "nccl" else "cpu"
    acc = torch.tensor(np.concatenate([z.sum(axis=0), [float(count)]]), dtype=torch.float64,
                       device=dev)
    if world > 1:
        dist.all_reduce(acc, group=group)
    acc = acc.cpu().numpy()
    return acc[:n] / acc[n], z, first
