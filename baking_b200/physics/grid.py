"""Dense background grid and its velocity update (the reference's ``physics/grid.py:4-38``).

Mechanics nodes are packed float4: ``node_pm[i] = (px, py, pz, m)`` and
``node_v[i] = (vx, vy, vz, 0)``; ``node_masses``, ``node_momenta`` and
``node_velocities`` are views with the reference's names and shapes.
"""

from __future__ import annotations

import torch

from .. import _lib


class GridState:
    def __init__(self, simulation_config, device_name="cuda", requires_grad=False):
        del requires_grad
        self.resolution = simulation_config.grid_resolution
        self.node_count = self.resolution ** 3
        self.node_pm = torch.zeros(self.node_count, 4, dtype=torch.float32, device=device_name)
        self.node_v = torch.zeros(self.node_count, 4, dtype=torch.float32, device=device_name)

    @property
    def node_masses(self):
        return self.node_pm[:, 3]

    @property
    def node_momenta(self):
        return self.node_pm[:, :3]

    @property
    def node_velocities(self):
        return self.node_v[:, :3]

    def Clear(self):
        self.node_pm.zero_()
        self.node_v.zero_()


def UpdateGrid(grid_state, simulation_config, time_step=None):
    """UpdateGrid (physics/grid.py:20-38) over the whole grid."""
    s = simulation_config
    gravity = (_lib.F32 * 3)(*s.gravity)
    _lib.call("bk_update_grid", s.grid_resolution, grid_state.node_pm.data_ptr(), grid_state.node_v.data_ptr(),
              s.boundary_cells, gravity, s.time_step if time_step is None else time_step,
              _lib.stream_handle())
