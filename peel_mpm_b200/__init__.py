"""B200-native (sm_100a) AnisoMPM substep with the reference solver's API.

    from peel_mpm_b200 import AnisoMPM, halfspace_collider, sphere_collider, grip_bc

The compute path is libpeelmpm.so (hand-written CUDA behind a C ABI, see
include/peelmpm.h), built in-tree by ``python -m peel_mpm_b200.build``.
Importing this package needs no GPU; constructing a solver needs an sm_100
device and the built library, and fails otherwise.
"""
from .anisompm import (AnisoMPM, Collider, ParticleGrip, bin_particles, grip_bc, halfspace_collider,
                       sphere_collider, sym_eig)
from .batched import BatchedAnisoMPM, partition_scenes

__all__ = ["AnisoMPM", "BatchedAnisoMPM", "Collider", "ParticleGrip", "bin_particles", "grip_bc",
           "halfspace_collider", "partition_scenes", "sphere_collider", "sym_eig"]
