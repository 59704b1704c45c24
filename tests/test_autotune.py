"""Autotuner logic on the CPU: the roofline fit of the reference's profiler
(src/profile.rs:137-183), the tensor-pipe crossover, and the fusion-width
choice from a pass-time table."""
import math

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
