"""Autotuner logic on the CPU: the roofline fit of the reference's profiler
(src/profile.rs:137-183), the tensor-pipe crossover, and the fusion-width
choice from a pass-time table."""
import math

import numpy as np

import pytest

from cast_simulator_b200 import autotune as A


def _probes(slope, peak, ks=range(1, 8), mode="f32"):
    out = []
    for k in ks:
        ai = A.dense_ai(k)
        g = min(slope * ai, peak)
        out.append(A.Probe(k, mode, ai, seconds=1.0, gflops_s=g, gib_s=g / ai))
    return out


def test_fit_recovers_two_segment_roofline():
    pr = _probes(100.0, 1600.0)
    slope, peak, xo = A.fit_roofline(pr)
    assert slope == pytest.approx(100.0) and peak == pytest.approx(1600.0)
    assert xo == pytest.approx(16.0)
    assert A.roofline_r2(pr, slope, peak) == pytest.approx(1.0)
    with pytest.raises(ValueError):
        A.fit_roofline([])


def test_tensor_probes_raise_the_crossover_for_wide_gates(cblib):
    pr = _probes(100.0, 1600.0)
    tensor = [A.Probe(5, "tc", 64.0, 1.0, 6000.0, 1.0), A.Probe(6, "tc", 128.0, 1.0, 9000.0, 1.0)]
    prof = A.profile_from_probes(pr, "f32", 26, tensor)
    assert prof.tensor_min_k == 5 and prof.tensor_gflops_s == pytest.approx(9000.0)
    assert prof.crossover_for(4) == pytest.approx(16.0)
    assert prof.crossover_for(6) == pytest.approx(90.0)
    assert A.profile_from_probes(pr, "f64", 26).crossover_for(6) == pytest.approx(16.0)


def test_engine_for():
    assert A.engine_for(6, "f32", True) == "tc"
    assert A.engine_for(4, "f32", True) == "f32"
    assert A.engine_for(6, "f64", True) == "f64"
    assert A.engine_for(6, "f32", False) == "f32"


def test_engine_for_sparse_gates():
    assert A.engine_for(6, "f64", False, sparse=True) == "sf64"
    assert A.engine_for(6, "f32", True, sparse=True) == "sf32"  # ahead of the tensor cores
    assert A.engine_for(4, "f32", True, sparse=True) == "f32"   # dense kernels below k = 5


def test_is_sparse_rule():
    rng = np.random.default_rng(0)
    assert A.is_sparse(A.monomial(5, rng))
    assert not A.is_sparse(A.monomial(4, rng))  # k < 5
    assert not A.is_sparse(A.haar(5, rng))
    blk = np.kron(np.eye(16), A.haar(2, rng))   # 4 nonzeros a row of 64
    assert A.is_sparse(blk)
    edge = np.kron(np.eye(4), A.haar(4, rng))   # 16 nonzeros a row of 64: the limit
    assert A.is_sparse(edge)
    dense = np.kron(np.eye(2), A.haar(5, rng))  # 32 nonzeros a row of 64
    assert not A.is_sparse(dense)
    tiny = A.monomial(5, rng) + 1e-16           # below ztol / 2^k: snapped to zero
    assert A.is_sparse(tiny)


def test_choose_fusion_prices_sparse_gates(cblib):
    """QFT-CX fuses into sparse blocks: with cheap sparse passes and dense wide
    passes priced high, the chooser still fuses wide."""
    from cast_simulator_b200.types import QuantumCircuit

    n = 14
    gates = QuantumCircuit.qft_cx(n).gates()
    tab = {(k, "f64"): 1.0 if k <= 4 else 3.0 for k in range(1, 8)}
    tab.update({(k, "sf64"): 1.1 for k in (5, 6, 7)})
    ch = A.choose_fusion(n, gates, "f64", A.PassTable(n, tab), ks=range(2, 7))
    assert ch.fusion_k >= 5
    without = A.choose_fusion(n, gates, "f64",
                              A.PassTable(n, {**tab, **{(k, "sf64"): 50.0 for k in (5, 6, 7)}}),
                              ks=range(2, 7))
    assert without.fusion_k <= 4


def _brickwork(n, depth):
    from cast_simulator_b200.types import QuantumCircuit

    return QuantumCircuit.brickwork(n, depth, 2024).gates()


def test_choose_fusion_prefers_the_fastest_predicted_engine(cblib):
    n = 16
    gates = _brickwork(n, 8)
    base = {(k, "f32"): 1.0 if k <= 4 else 2.0 ** (k - 3) for k in range(1, 8)}
    cheap_tc = A.PassTable(n, {**base, (5, "tc"): 1.2, (6, "tc"): 1.3})
    ch = A.choose_fusion(n, gates, "f32", cheap_tc)
    assert ch.split_precision and ch.fusion_k >= 5
    dear_tc = A.PassTable(n, {**base, (5, "tc"): 9.0, (6, "tc"): 9.0})
    ch2 = A.choose_fusion(n, gates, "f32", dear_tc)
    assert not ch2.split_precision and ch2.fusion_k <= 4
    # predictions scale with the statevector size (memory-bound passes)
    assert dear_tc.predict(3, "f32", n + 2) == pytest.approx(4.0)
    with pytest.raises(KeyError):
        dear_tc.predict(7, "tc", n)
    assert all(math.isfinite(c["predicted_s"]) for c in ch.candidates)
