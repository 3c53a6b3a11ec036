"""Particle state containers (the reference's ``physics/state.py:6-46``).

Same dataclasses and field names; the arrays are CUDA torch tensors in the
plane layout of :mod:`baking_b200.arrays` ((n, 3) / (n, 3, 3) views).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .. import arrays


@dataclass
class ParticleState:
    particle_positions: torch.Tensor
    particle_velocities: torch.Tensor
    deformation_gradients: torch.Tensor
    affine_velocities: torch.Tensor
    material_state: object = None
    transport_state: object = None


@dataclass
class ParticleData:
    particle_masses: torch.Tensor
    reference_volumes: torch.Tensor
    particle_count: int


def AllocateState(particle_count, device_name="cuda", requires_grad=False):
    del requires_grad  # gradients come from the hand-written adjoint, not autograd on these arrays
    return ParticleState(arrays.vec3s(particle_count, device=device_name),
                         arrays.vec3s(particle_count, device=device_name),
                         arrays.mat33s(particle_count, device=device_name),
                         arrays.mat33s(particle_count, device=device_name))


def CreateParticleState(particle_samples, device_name="cuda", initial_velocity=(0.0, 0.0, 0.0),
                        requires_grad=False):
    count = len(particle_samples.particle_positions)
    v0 = np.asarray(initial_velocity, dtype=np.float32)
    if v0.shape != (3,) or not np.isfinite(v0).all():
        raise ValueError("initial_velocity must have three finite components")
    state = AllocateState(count, device_name, requires_grad)
    arrays.assign(state.particle_positions, particle_samples.particle_positions.astype(np.float32))
    state.particle_velocities.copy_(torch.as_tensor(v0, device=state.particle_velocities.device))
    state.deformation_gradients.copy_(torch.eye(3, device=state.deformation_gradients.device))
    data = ParticleData(arrays.from_numpy(np.asarray(particle_samples.particle_masses, np.float32), "f4", device_name),
                        arrays.from_numpy(np.asarray(particle_samples.reference_volumes, np.float32), "f4",
                                          device_name), count)
    return state, data
