"""P2G scatter and G2P gather (the reference's ``physics/transfer.py:36-109``) on the device."""

from __future__ import annotations

from .. import _lib, arrays


def _origin(origin):
    return (_lib.F32 * 3)(*origin)


def ParticleToGrid(particle_positions, particle_velocities, affine_velocities, kirchhoff_stresses, particle_masses,
                   reference_volumes, grid_state, grid_origin, grid_spacing, grid_resolution, time_step,
                   error_flags):
    """Adds w m and w (m v + (m C - dt V0 4/dx^2 tau)(x_i - x_p)) into ``grid_state.node_pm``."""
    n = particle_positions.shape[0]
    pitch = arrays.common_pitch(particle_positions, particle_velocities, affine_velocities, kirchhoff_stresses)
    _lib.call("bk_particle_to_grid", n, pitch, arrays.ptr(particle_positions), arrays.ptr(particle_velocities),
              arrays.ptr(affine_velocities), arrays.ptr(kirchhoff_stresses), arrays.ptr(particle_masses),
              arrays.ptr(reference_volumes), grid_state.node_pm.data_ptr(), _origin(grid_origin), grid_spacing,
              grid_resolution, time_step, error_flags.data_ptr(), _lib.stream_handle())


def GridToParticle(input_positions, input_gradients, grid_state, output_positions, output_velocities,
                   output_affines, output_gradients, grid_origin, grid_spacing, grid_resolution, time_step,
                   error_flags):
    n = input_positions.shape[0]
    pitch = arrays.common_pitch(input_positions, input_gradients, output_positions, output_velocities,
                                output_affines, output_gradients)
    _lib.call("bk_grid_to_particle", n, pitch, arrays.ptr(input_positions), arrays.ptr(input_gradients),
              grid_state.node_v.data_ptr(), arrays.ptr(output_positions), arrays.ptr(output_velocities),
              arrays.ptr(output_affines), arrays.ptr(output_gradients), _origin(grid_origin), grid_spacing,
              grid_resolution, time_step, error_flags.data_ptr(), _lib.stream_handle())
