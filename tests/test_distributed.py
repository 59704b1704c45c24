"""Sharded statevector with qubit-swap exchanges: the swap planner (greedy and
look-ahead), the index permutation, and world-size 2 and 4 runs over gloo on
CPU (one process per rank, the oracle as the local gate applier) against the
oracle's unsharded run, with exchanges streamed through small staging chunks."""
import os
import socket

import numpy as np
import pytest

from cast_simulator_b200 import distributed as D


def test_swap_plan():
    assert D.swap_plan((0, 3), 6) == []
    assert D.swap_plan((2, 7), 6) == [(7, 5)]
    assert D.swap_plan((5, 6, 7), 6) == [(6, 4), (7, 3)]
    assert D.swap_plan((6,), 6, in_use={5}) == [(6, 4)]
    with pytest.raises(ValueError, match="wider"):
        D.swap_plan((0, 1, 2), 2)


def test_swap_plan_priority_and_next_uses():
    # look-ahead: evict the local position whose logical qubit is used last
    nxt = D.next_uses([(0, 1), (2,), (1, 5), (0,)], 6)
    assert nxt[0] == {2: 1, 1: 2, 5: 2, 0: 3}
    assert nxt[1] == {1: 2, 5: 2, 0: 3} and nxt[3] == {}
    prio = {5: 1.0, 4: 7.0, 3: float("inf"), 2: 3.0, 1: 0.0, 0: 2.0}
    assert D.swap_plan((6,), 6, priority=prio.get) == [(6, 3)]
    assert D.swap_plan((6, 7), 6, priority=prio.get) == [(6, 3), (7, 4)]
    # ties go to the highest position
    assert D.swap_plan((6,), 6, priority=lambda p: 1.0) == [(6, 5)]


def test_permute_bits():
    idx = np.arange(8)
    assert np.array_equal(D.permute_bits(idx, [0, 1, 2]), idx)
    assert np.array_equal(D.permute_bits(idx, [2, 1, 0]), [0, 4, 2, 6, 1, 5, 3, 7])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _circuit(n, seed):
    rng = np.random.default_rng(seed)
    gates = []
    for _ in range(40):
        k = int(rng.integers(1, 4))
        q = [int(x) for x in rng.choice(n, size=k, replace=False)]  # arbitrary order
        z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
        gates.append((np.linalg.qr(z)[0], q))
    return gates


def _worker(rank, world, port, n, seed, out_dir, chunk=1 << 24, lookahead=False):
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from cast_simulator_b200 import distributed as D
    from cast_simulator_b200.types import _canonicalize
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        def apply_local(shard, m, qs):
            mm, srt = _canonicalize(np.asarray(m), list(qs))
            O.apply_gate(shard.numpy(), mm, srt)  # in place on the shard's memory

        n_local = n - (world.bit_length() - 1)
        sv = D.ShardedStatevector(n, torch.zeros(1 << n_local, dtype=torch.complex128), apply_local,
                                  chunk_amps=chunk)
        sv.set_zero()
        if lookahead:
            class G:
                def __init__(self, m, q):
                    self._m, self._q = m, q

                def matrix(self):
                    return self._m

                def qubits(self):
                    return self._q

            sv.apply_circuit([G(m, q) for m, q in _circuit(n, seed)])
        else:
            for m, q in _circuit(n, seed):
                sv.apply(m, q)
        full = sv.gather()
        z = sv.expectation_z()
        if rank == 0:
            np.save(os.path.join(out_dir, "state.npy"), full)
            np.save(os.path.join(out_dir, "z.npy"), z)
            np.save(os.path.join(out_dir, "ex.npy"), np.array([sv.n_exchanges, sv.exchanged_amps]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,chunk,lookahead", [(2, 1 << 24, False), (4, 1 << 24, False),
                                                   (2, 4, False), (4, 2, True), (4, 16, True)])
def test_sharded_matches_oracle(oracle, tmp_path, world, chunk, lookahead):
    """Whole-half exchanges, exchanges streamed through staging chunks smaller
    than one run and larger than one run, and the look-ahead planner: all give
    the oracle's state and <Z>."""
    import torch.multiprocessing as mp

    n, seed = 8, 11 + world
    mp.start_processes(_worker, args=(world, _free_port(), n, seed, str(tmp_path), chunk, lookahead),
                       nprocs=world, join=True, start_method="spawn")
    got = np.load(tmp_path / "state.npy")
    gates = []
    from cast_simulator_b200.types import _canonicalize

    for m, q in _circuit(n, seed):
        mm, srt = _canonicalize(m, q)
        gates.append((mm, srt))
    ref = oracle.simulate(n, gates)
    assert np.max(np.abs(got - ref)) < 1e-12
    p = np.abs(ref) ** 2
    idx = np.arange(1 << n)
    z_ref = np.array([1 - 2 * p[(idx >> q) & 1 == 1].sum() for q in range(n)])
    assert np.max(np.abs(np.load(tmp_path / "z.npy") - z_ref)) < 1e-12
    ex, amps = (int(x) for x in np.load(tmp_path / "ex.npy"))
    assert ex > 0  # the circuit did cross shards
    n_local = n - (world.bit_length() - 1)
    assert amps == ex * (1 << (n_local - 1))  # each exchange moved half a shard


def test_lookahead_needs_no_more_exchanges():
    """Belady's rule on a host model of the planner: over random circuits the
    look-ahead choice never makes more exchanges than the greedy one, and makes
    fewer on most."""
    rng = np.random.default_rng(3)
    fewer = 0
    for trial in range(30):
        n, n_local = 12, 9
        circ = []
        for _ in range(120):
            k = int(rng.integers(1, 4))
            circ.append(tuple(int(x) for x in rng.choice(n, size=k, replace=False)))

        def count(lookahead):
            perm = list(range(n))
            nxt = D.next_uses(circ, n)
            swaps = 0
            for i, qs in enumerate(circ):
                phys = tuple(perm[q] for q in qs)
                prio = None
                if lookahead:
                    at = {p: lq for lq, p in enumerate(perm)}
                    prio = lambda pos, i=i, at=at: nxt[i].get(at[pos], float("inf"))  # noqa: E731
                for g, l in D.swap_plan(phys, n_local, priority=prio):
                    a, b = perm.index(g), perm.index(l)
                    perm[a], perm[b] = l, g
                    swaps += 1
            return swaps

        greedy, ahead = count(False), count(True)
        assert ahead <= greedy
        fewer += ahead < greedy
    assert fewer >= 20


def test_trajectory_range_partition():
    for n_traj in (0, 1, 7, 4096):
        for world in (1, 2, 3, 8):
            parts = [D.trajectory_range(n_traj, world, r) for r in range(world)]
            assert sum(c for _, c in parts) == n_traj
            nxt = 0
            for first, count in parts:
                assert first == nxt  # contiguous, in rank order
                nxt = first + count
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
    with pytest.raises(ValueError):
        D.trajectory_range(10, 2, 2)


class _IndexedProgram:
    """Stands in for a TrajectoryProgram: row j of a run is a fixed function of
    the global trajectory index first + j (as the device kernel's Philox streams
    are)."""

    n = 5

    def run(self, count, seed, stream=None, first=0):
        idx = np.arange(first, first + count, dtype=np.float64)[:, None]
        q = np.arange(self.n)[None, :]
        return np.cos(0.37 * idx * (q + 1) + seed), np.zeros(count, dtype=np.uint32)


def _traj_worker(rank, world, port, n_traj, out_dir):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from cast_simulator_b200 import distributed as D
    from tests.test_distributed import _IndexedProgram

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mean, rows, first = D.run_trajectories_sharded(_IndexedProgram(), n_traj, 3)
        np.save(os.path.join(out_dir, f"mean{rank}.npy"), mean)
        np.save(os.path.join(out_dir, f"rows{rank}.npy"), rows)
        np.save(os.path.join(out_dir, f"first{rank}.npy"), np.array([first]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n_traj", [(2, 101), (3, 2)])
def test_sharded_trajectories_equal_one_batch(tmp_path, world, n_traj):
    """Ranges over gloo ranks reproduce the single batch row for row and the
    all-reduced mean equals its mean (a rank may get no trajectories)."""
    import torch.multiprocessing as mp

    mp.start_processes(_traj_worker, args=(world, _free_port(), n_traj, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    full, _ = _IndexedProgram().run(n_traj, 3)
    rows = np.concatenate([np.load(tmp_path / f"rows{r}.npy") for r in range(world)])
    assert np.array_equal(rows, full)
    for r in range(world):
        assert np.allclose(np.load(tmp_path / f"mean{r}.npy"), full.mean(axis=0), atol=1e-14)
