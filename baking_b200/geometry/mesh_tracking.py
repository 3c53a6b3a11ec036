"""Rebuild tet-mesh vertices from particle x and F (the reference's ``geometry/mesh_tracking.py:13-81``).

Each vertex is bound to the particles sampled in its incident tets; particle p
predicts x_v = x_p + F_p (X_v - X_p) and the predictions are blended with
reference-volume weights (as deviations from the first binding, the anchor).
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib, arrays
from .sampling import MeshBindingTables_build


class ParticleMeshBinding:
    def __init__(self, tet_mesh, particle_samples, device_name="cuda"):
        tables = MeshBindingTables_build(tet_mesh, particle_samples)
        self.tables = tables
        self.unmapped_vertex_count = tables.unmapped_vertex_count
        self.vertex_count = len(tet_mesh.vertex_positions)
        self.reference_vertices = arrays.from_numpy(tet_mesh.vertex_positions.astype(np.float32), "f4", device_name)
        self.binding_offsets = torch.as_tensor(tables.binding_offsets, device=device_name)
        self.binding_particles = torch.as_tensor(tables.binding_particles, device=device_name)
        self.binding_weights = torch.as_tensor(tables.binding_weights.astype(np.float32), device=device_name)
        self.reference_offsets = arrays.from_numpy(tables.reference_offsets.astype(np.float32), "f4", device_name)

    def Reconstruct(self, particle_state, output_vertices):
        x = particle_state.particle_positions
        pitch = arrays.common_pitch(x, particle_state.deformation_gradients)
        _lib.call("bk_reconstruct_mesh_vertices", self.vertex_count, pitch, arrays.ptr(x),
                  arrays.ptr(particle_state.deformation_gradients), arrays.layout_pitch(output_vertices),
                  arrays.ptr(self.reference_vertices), self.binding_offsets.data_ptr(),
                  self.binding_particles.data_ptr(), self.binding_weights.data_ptr(),
                  arrays.layout_pitch(self.reference_offsets), arrays.ptr(self.reference_offsets),
                  arrays.ptr(output_vertices), _lib.stream_handle())
