"""cast_simulator_b200: a B200-native (sm_100a) gate-application engine behind
the CUDA-backend C ABI of narix10yc/cast_simulator (CAST).

Layers (bottom up):
  * ``libcast_b200.so`` (csrc/): hand-written sm_100a kernels, the drop-in
    ``ffi_cuda.h`` C ABI and the ``cast_b200.h`` extensions;
  * ``cuda``: CudaKernelGenSpec / CudaStatevector / CudaKernelManager over the ABI;
  * ``types`` / ``fusion``: gates, noise, circuits, circuit graph, fusion and
    cost models (host-side, mirroring CAST's Rust types);
  * ``simulator``: Simulator.simulate / bench, QuantumState;
  * ``trajectory`` / ``serving``: batched noisy trajectories and the
    continuous-batching request loop.
"""
from .types import NoiseModel, QuantumCircuit, QuantumGate, SplitMix64  # noqa: F401
from .fusion import (  # noqa: F401
    CircuitGraph,
    FusionConfig,
    HardwareAdaptiveCostModel,
    HardwareProfile,
    SizeOnlyCostModel,
    optimize,
)

__all__ = [
    "NoiseModel", "QuantumCircuit", "QuantumGate", "SplitMix64", "CircuitGraph", "FusionConfig",
    "HardwareAdaptiveCostModel", "HardwareProfile", "SizeOnlyCostModel", "optimize",
]
