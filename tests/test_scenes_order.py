"""Host side of the particle order, no GPU: the generated scenes list particles grouped by
quadratic stencil base, and scenes.permuted reorders every per-particle sample array and
per-particle gas source rate together and refuses non-permutations."""
import numpy as np
import pytest

from baking_b200.scenes import dough_ball, permuted


def stencil_bases(points, dx):
    return np.floor(points / dx - 0.5).astype(np.int64)


def test_generated_scene_groups_particles_by_stencil_base():
    scene = dough_ball(32, 3000, seed=3)
    b = stencil_bases(scene.samples.particle_positions, scene.simulation.grid_spacing)
    key = (b[:, 0] * 1024 + b[:, 1]) * 1024 + b[:, 2]
    # each base appears as one contiguous run
    starts = np.flatnonzero(np.diff(key) != 0) + 1
    runs = np.split(key, starts)
    assert len({int(r[0]) for r in runs}) == len(runs)


def test_permuted_moves_every_per_particle_array_together():
    scene = dough_ball(32, 3000, seed=5)
    n = len(scene.samples.particle_positions)
    order = np.random.default_rng(2).permutation(n)
    out = permuted(scene, order)
    np.testing.assert_array_equal(out.samples.particle_positions, scene.samples.particle_positions[order])
    np.testing.assert_array_equal(out.samples.reference_volumes, scene.samples.reference_volumes[order])
    np.testing.assert_array_equal(out.samples.particle_masses, scene.samples.particle_masses[order])
    np.testing.assert_array_equal(out.samples.source_tets, scene.samples.source_tets[order])
    assert scene.gas_source_rates is not None and len(scene.gas_source_rates) == n
    np.testing.assert_array_equal(out.gas_source_rates, scene.gas_source_rates[order])
    assert out.tet_mesh is scene.tet_mesh and out.simulation == scene.simulation
    # the original scene is untouched
    assert not np.array_equal(scene.samples.particle_positions, out.samples.particle_positions)


def test_permuted_rejects_non_permutations():
    scene = dough_ball(32, 2000, seed=5)
    n = len(scene.samples.particle_positions)
    with pytest.raises(ValueError):
        permuted(scene, np.zeros(n, dtype=np.int64))
    with pytest.raises(ValueError):
        permuted(scene, np.arange(n - 1))


def test_permutation_table_takes_plane_layout_arrays_only():
    """SortParticles hands plane-layout arrays ((n, 3) with strides (1, pitch), (n, 3, 3) with
    strides (1, 3 pitch, pitch)) to bk_permute_particles and row-major ones to torch."""
    import ctypes
    import torch
    from baking_b200 import _lib, arrays
    from baking_b200.physics.mpm import _plane_layout
    assert _plane_layout(arrays.vec3s(100, device="cpu")) and _plane_layout(arrays.mat33s(100, device="cpu"))
    assert not _plane_layout(torch.zeros(100, 3)) and not _plane_layout(torch.zeros(100, 3, 3))
    assert ctypes.sizeof(_lib.BkParticleArray) == 24  # void*, int64_t, int32_t, int32_t
