"""nbb -- B200-native Barnes-Hut N-body step (Python side of libnbb.so).

The package mirrors the public API of sytrams/AMSC-Nbody's hot path
(Simulation, SimulationConfig, BarnesHutParameters,
computeBarnesHutAcceleration, leapfrog integrator) over the C ABI declared in
include/nbb.h.  All arithmetic runs in the CUDA library; this package only
marshals arguments.
"""
from ._lib import (POTENTIAL_DIRECT, POTENTIAL_NONE, POTENTIAL_TREE, PRECISION_FP64, PRECISION_MIXED, DeviceError, DomainError, InvalidArgument,
                   LogicError, NbbError, NoDevice, OverflowErrorNbb, load)
from .api import (G_SI, BarnesHutParameters, ConservationMonitor, EnsembleSimulation, Simulation, SimulationConfig, compute_accelerations,
                  compute_direct_accelerations, computeBarnesHutAcceleration, direct_rollout_adjoint,
                  frozen_rollout, kernel_launch_count, measure_fma_tflops,
                  leapfrog_kick, leapfrog_kick_drift, node_capacity, octree_from_keys, radix_tree)
from .ics import ParticleData

__all__ = [
    "POTENTIAL_DIRECT", "POTENTIAL_NONE", "POTENTIAL_TREE", "PRECISION_FP64", "PRECISION_MIXED", "DeviceError", "DomainError", "InvalidArgument",
    "LogicError", "NbbError", "NoDevice", "OverflowErrorNbb", "load", "G_SI",
    "BarnesHutParameters", "ConservationMonitor", "EnsembleSimulation", "Simulation", "SimulationConfig", "compute_accelerations",
    "compute_direct_accelerations", "computeBarnesHutAcceleration", "direct_rollout_adjoint",
    "frozen_rollout", "kernel_launch_count", "measure_fma_tflops",
    "leapfrog_kick", "leapfrog_kick_drift", "node_capacity", "octree_from_keys", "radix_tree",
    "ParticleData",
]
