"""B200-native (sm_100a) implementation of HeddleMD's per-timestep
force-and-constraint path: packed neighbour list, LJ + erfc real-space pair
kernel, SPME spread / FFT / convolution / gather, SETTLE / SHAKE, deterministic
fixed-point and FP64 reductions, behind a C ABI (include/heddle_b200.h)."""

from ._native import HeddleError, load  # noqa: F401
from .api import (  # noqa: F401
    Barostat,
    Batch,
    Constraints,
    Context,
    ForceField,
    Integrator,
    HarmonicAngleParams,
    HarmonicBondParams,
    LennardJonesParams,
    Minimizer,
    PeriodicDihedralParams,
    PotentialRegistry,
    PressureCoupling,
    ShakeMLP,
    SpmeParams,
    System,
    Thermostat,
)

__all__ = [
    "Context", "System", "ForceField", "Constraints", "Integrator", "Barostat", "Batch",
    "PotentialRegistry", "LennardJonesParams", "SpmeParams", "HarmonicBondParams",
    "HarmonicAngleParams", "PeriodicDihedralParams", "ShakeMLP", "Thermostat",
    "PressureCoupling", "Minimizer", "HeddleError", "load",
]
