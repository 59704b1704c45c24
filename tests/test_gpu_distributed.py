"""The sharded statevector's GPU applier (device kernels through the C ABI on a
torch-allocated shard, on torch's current stream) at world size 1; the
multi-rank exchanges are covered by tests/test_distributed.py over gloo."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_cuda_applier_single_rank(cblib, oracle):
    import torch

    from cast_simulator_b200 import distributed as D

    n = 12
    rng = np.random.default_rng(4)
    gates = []
    for _ in range(30):
        k = int(rng.integers(1, 5))
        q = [int(x) for x in rng.choice(n, size=k, replace=False)]
        z = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
        gates.append((np.linalg.qr(z)[0], q))
    for dtype, prec, tol in ((torch.complex128, 1, 1e-10), (torch.complex64, 0, 1e-5)):
        sv = D.ShardedStatevector(n, torch.zeros(1 << n, dtype=dtype, device="cuda"),
                                  D.cuda_apply_local(prec))
        sv.set_zero()
        for m, q in gates:
            sv.apply(m, q)
        torch.cuda.synchronize()
        got = sv.gather()
        from cast_simulator_b200.types import _canonicalize

        ref = oracle.simulate(n, [_canonicalize(m, q) for m, q in gates])
        assert np.max(np.abs(got - ref)) < tol
        p = np.abs(ref) ** 2
        idx = np.arange(1 << n)
        z_ref = np.array([1 - 2 * p[(idx >> q) & 1 == 1].sum() for q in range(n)])
        assert np.max(np.abs(sv.expectation_z() - z_ref)) < tol


def test_cuda_applier_apply_circuit_single_rank(cblib, oracle):
    """apply_circuit (the look-ahead planner's entry point) through the device
    kernels at world size 1: no exchanges, the oracle's state."""
    import torch

    from cast_simulator_b200 import distributed as D
    from cast_simulator_b200.fusion import FusionConfig, optimize_native
    from cast_simulator_b200.types import QuantumCircuit

    n = 14
    circ = QuantumCircuit.brickwork(n, 6, 9)
    fused = optimize_native(n, circ.gates(), FusionConfig.size_only(4)).gates()
    sv = D.ShardedStatevector(n, torch.zeros(1 << n, dtype=torch.complex128, device="cuda"),
                              D.cuda_apply_local(1))
    sv.set_zero()
    sv.apply_circuit(fused)
    torch.cuda.synchronize()
    ref = oracle.simulate(n, [(g.matrix(), g.qubits()) for g in circ.gates()])
    assert np.max(np.abs(sv.gather() - ref)) < 1e-10
    assert sv.n_exchanges == 0
