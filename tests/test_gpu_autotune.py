"""Autotuner on the device: gate timings, the fitted profile with the
tensor-pipe crossover, and the fusion choice from measured pass times."""
import pytest

pytestmark = pytest.mark.gpu


def test_tensor_cores_beat_cuda_cores_on_wide_gates(cblib):
    from cast_simulator_b200 import autotune as A

    t_tc = A.time_gate(24, 6, "tc")
    t_f32 = A.time_gate(24, 6, "f32")
    assert 0 < t_tc < t_f32


def test_profile_and_choice(cblib):
    from cast_simulator_b200 import autotune as A
    from cast_simulator_b200.types import QuantumCircuit

    prof = A.measure_profile(20, "f32", ks=range(1, 7), reps=2)
    assert prof.peak_bw_gib_s > 0 and prof.bw_slope > 0 and prof.peak_gflops_s > 0
    assert prof.tensor_min_k == 5 and prof.tensor_gflops_s > 0
    assert prof.crossover_for(6) > 0 and prof.config["r2"] <= 1.0
    tab = A.measure_pass_table(20, "f32", ks=range(1, 7), reps=2)
    gates = QuantumCircuit.brickwork(22, 8, 5).gates()
    ch = A.choose_fusion(22, gates, "f32", tab, ks=range(2, 7))
    assert 2 <= ch.fusion_k <= 6
    assert ch.predicted_s <= min(c["predicted_s"] for c in ch.candidates) + 1e-15


def test_trajectory_tuning_picks_the_fastest_shape(cblib):
    from cast_simulator_b200 import autotune as A
    from cast_simulator_b200.types import QuantumCircuit

    circ = QuantumCircuit.brickwork(12, 6, 3, depolarizing=1e-3, damping=5e-4)
    ch = A.tune_trajectories(circ, n_traj=512, ks=(2, 3), threads=(512, 1024), ctas=(0, 64))
    assert len(ch.candidates) == 8
    assert ch.traj_per_s == max(c["traj_per_s"] for c in ch.candidates) > 0
    assert ch.fusion_k in (2, 3) and ch.threads in (512, 1024) and ch.max_ctas in (0, 64)
