"""Rebuild tet-mesh vertices from particle x and F (the reference's ``geometry/mesh_tracking.py:13-81``).

Each vertex is bound to the particles sampled in its incident tets; particle p
predicts x_v = x_p + F_p (X_v - X_p) and the predictions are blended with
reference-volume weights (as deviations from the first binding, the anchor).
"""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import torch

from .. import _lib, arrays
from .sampling import MeshBindingTables_build


class ParticleMeshBinding:
    def __init__(self, tet_mesh, particle_samples, device_name="cuda"):
        tables = MeshBindingTables_build(tet_mesh, particle_samples)
        self._tables = tables
        self._host_particles_stale = False
        self.unmapped_vertex_count = tables.unmapped_vertex_count
        self.vertex_count = len(tet_mesh.vertex_positions)
        self.reference_vertices = arrays.from_numpy(tet_mesh.vertex_positions.astype(np.float32), "f4", device_name)
        self.binding_offsets = torch.as_tensor(tables.binding_offsets, device=device_name)
        self.binding_particles = torch.as_tensor(tables.binding_particles, device=device_name)
        self.binding_weights = torch.as_tensor(tables.binding_weights.astype(np.float32), device=device_name)
        self.reference_offsets = arrays.from_numpy(tables.reference_offsets.astype(np.float32), "f4", device_name)

    @property
    def tables(self):
        """The host binding tables; their particle indices follow a renumbering of the device
        ones (``RenumberParticles``) when next read."""
        if self._host_particles_stale:
            self._tables = replace(self._tables, binding_particles=self.binding_particles.cpu().numpy())
            self._host_particles_stale = False
        return self._tables

    def RenumberParticles(self, new_index):
        """After a particle reordering: binding particle p becomes ``new_index[p]`` (device)."""
        t = self.binding_particles
        t.copy_(torch.where(t >= 0, new_index[t.clamp(min=0).long()].to(t.dtype), t))
        self._host_particles_stale = True

    def Reconstruct(self, particle_state, output_vertices):
        x = particle_state.particle_positions
        pitch = arrays.common_pitch(x, particle_state.deformation_gradients)
        _lib.call("bk_reconstruct_mesh_vertices", self.vertex_count, pitch, arrays.ptr(x),
                  arrays.ptr(particle_state.deformation_gradients), arrays.layout_pitch(output_vertices),
                  arrays.ptr(self.reference_vertices), self.binding_offsets.data_ptr(),
                  self.binding_particles.data_ptr(), self.binding_weights.data_ptr(),
                  arrays.layout_pitch(self.reference_offsets), arrays.ptr(self.reference_offsets),
                  arrays.ptr(output_vertices), _lib.stream_handle())
