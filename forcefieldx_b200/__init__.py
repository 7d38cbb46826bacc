"""B200-native AMOEBA polarizable energy and gradient (Force Field X hot path).

The compute path is libffxcuda.so (hand-written sm_100a CUDA behind the C ABI in
include/ffxcuda.h); this package holds the host-side mirror of the reference's
ForceFieldEnergy / ParticleMeshEwald interface and the system builders.
"""
from .system import (AmoebaParams, AmoebaSystem, water_box, water_params,  # noqa: F401
                     PRECISION_FP64, PRECISION_MIXED, POLAR_MUTUAL, POLAR_DIRECT, POLAR_NONE)
