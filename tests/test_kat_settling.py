"""Known answers of the reference's geometry and settling tests.

Restates tests/test_mesh_processing.py:8-54, tests/test_sphere.py:185-221 (mesh part),
tests/test_settling.py:173-224 and tests/test_auto_settling.py:243-298 of the reference.
Settling runs on the device; the oracle restates fixed-duration settling only.
"""
from dataclasses import replace

import numpy as np
import pytest

from baking_b200.config import TransportConfig
from baking_b200.geometry import (ComputeSignedVolumes, CreateDemoMesh, CreateSphereMesh, SampleParticles,
                                  ValidateTetMesh)
from tests.kat_api import ENGINES
from tests.scenes import assign, build_transport, to_np


def test_demo_volume_and_sampling():
    mesh = CreateDemoMesh(2)
    np.testing.assert_allclose(mesh.reference_volumes.sum(), 0.3 ** 3)
    assert np.all(ComputeSignedVolumes(mesh.vertex_positions, mesh.tet_indices) > 0.0)
    samples = SampleParticles(mesh, 1000.0, particles_per_tet=4)
    np.testing.assert_allclose(samples.reference_volumes.sum(), 0.3 ** 3)
    np.testing.assert_allclose(samples.particle_masses.sum(), 27.0)
    for t in range(len(mesh.tet_indices)):
        corners = mesh.vertex_positions[mesh.tet_indices[t]]
        pts = samples.particle_positions[samples.source_tets == t]
        bary = np.linalg.solve((corners[1:] - corners[0]).T, (pts - corners[0]).T).T
        assert np.all(bary >= 0.0) and np.all(bary.sum(axis=1) <= 1.0)


def test_invalid_mesh_rejected():
    mesh = CreateDemoMesh(1)
    with pytest.raises(ValueError, match="repeated"):
        ValidateTetMesh(mesh.vertex_positions, np.array([[0, 0, 1, 2]]))
    with pytest.raises(ValueError, match="degenerate"):
        ValidateTetMesh(np.zeros((4, 3)), np.array([[0, 1, 2, 3]]))


def test_automatic_sampling_and_limit():
    mesh = CreateDemoMesh(1)
    samples = SampleParticles(mesh, 1000.0, target_volume=0.001)
    assert len(samples.particle_positions) >= 24
    np.testing.assert_allclose(samples.reference_volumes.sum(), 0.027)
    with pytest.raises(ValueError, match="max_particles"):
        SampleParticles(mesh, 1000.0, target_volume=1.0e-12)


def test_sphere_boundary_volume():
    from itertools import combinations
    mesh = CreateSphereMesh()
    # Boundary faces are those used by one tet; their vertices lie on the sphere.
    faces = np.sort(np.concatenate([mesh.tet_indices[:, list(c)] for c in combinations(range(4), 3)]), axis=1)
    unique, counts = np.unique(faces, axis=0, return_counts=True)
    boundary_vertices = np.unique(unique[counts == 1])
    np.testing.assert_allclose(np.linalg.norm(mesh.vertex_positions[boundary_vertices], axis=1), 0.1, atol=1e-12)
    np.testing.assert_allclose(mesh.vertex_positions.min(axis=0), -0.1, atol=1e-12)
    np.testing.assert_allclose(mesh.vertex_positions.max(axis=0), 0.1, atol=1e-12)
    assert np.all(ComputeSignedVolumes(mesh.vertex_positions, mesh.tet_indices) > 0)
    np.testing.assert_allclose(mesh.reference_volumes.sum(), 4 * np.pi * 0.1 ** 3 / 3, rtol=0.01)


def resting(engine, history=False):
    sim = build_transport(engine, TransportConfig(enabled=True, settling_duration_s=.0004), history=history, gas=True)
    sim.simulation_config = replace(sim.simulation_config, gravity=(0., -9.81, 0.))
    sim.material.simulation_config = sim.simulation_config
    return sim


@pytest.mark.parametrize("engine", ENGINES)
def test_rest_is_isothermal_mass_conserving_and_falls_then_heats(engine):
    sim = resting(engine, history=engine != "oracle")
    initial = sim.current_state
    water = to_np(initial.transport_state.water_masses).copy()
    gas = to_np(initial.material_state.gas_moles).copy()
    y = to_np(initial.particle_positions)[:, 1].mean()
    for _ in range(4):
        sim.Step()
    settled = sim.current_state
    np.testing.assert_array_equal(to_np(settled.transport_state.water_masses), water)
    np.testing.assert_array_equal(to_np(settled.material_state.gas_moles), gas)
    np.testing.assert_allclose(to_np(settled.transport_state.temperatures), 293.15, atol=1e-12)
    np.testing.assert_array_equal(to_np(settled.transport_state.water_losses), 0.)
    np.testing.assert_array_equal(to_np(settled.transport_state.heat_exchanges), 0.)
    assert to_np(settled.particle_positions)[:, 1].mean() < y
    assert to_np(settled.particle_velocities)[:, 1].mean() < 0
    velocity = to_np(settled.particle_velocities).copy()
    sim.Step()
    assert to_np(sim.current_state.transport_state.temperatures).max() > 293.15
    assert to_np(sim.current_state.material_state.gas_moles).min() > gas.min()
    assert to_np(sim.current_state.particle_velocities)[:, 1].mean() < velocity[:, 1].mean()
    if engine != "oracle":
        assert sim.baking_time == sim.simulation_config.time_step
        assert len(sim.state_history) == 6 and sim.state_history[4] is settled


@pytest.mark.gpu
def test_zero_rest_preserves_legacy_and_duration_rounding():
    sim = resting("cuda")
    sim.transport.config = replace(sim.transport.config, settling_duration_s=.00041)
    assert sim.settling_steps == 5
    sim.transport.config = replace(sim.transport.config, settling_duration_s=0.)
    assert sim.settling_steps == 0
    sim.Step()
    assert to_np(sim.current_state.transport_state.temperatures).max() > 293.15


def auto(history=False, gravity=(0., 0., 0.)):
    config = TransportConfig(enabled=True, settling_duration_s=.002, settling_auto=True,
                             settling_min_duration_s=.0002, settling_hold_duration_s=.0003,
                             settling_speed_tolerance=1e-4, settling_rate_tolerance=.01)
    sim = build_transport("cuda", config, history=history, gas=True)
    sim.simulation_config = replace(sim.simulation_config, gravity=gravity)
    sim.material.simulation_config = sim.simulation_config
    return sim


@pytest.mark.gpu
def test_quiet_confirmation_then_baking_and_reset():
    sim = auto(history=True)
    initial = sim.current_state
    for _ in range(4):
        sim.Step()
        assert sim.IsSettling and sim.baking_time == 0
        np.testing.assert_allclose(to_np(sim.current_state.transport_state.temperatures), 293.15, atol=1e-12)
    sim.Step()
    assert not sim.IsSettling and sim.settling_reason == "quasi_static"
    assert sim.settling_steps == 5 and sim.baking_time == 0
    settled = sim.current_state
    sim.Step()
    assert sim.baking_steps == 1 and sim.baking_time == sim.simulation_config.time_step
    assert to_np(sim.current_state.transport_state.temperatures).max() > 293.15
    assert sim.state_history[0] is initial and sim.state_history[5] is settled
    sim.Reset()
    assert sim.IsSettling and sim.settling_quiet_steps == 0 and sim.baking_steps == 0


@pytest.mark.gpu
def test_moving_object_times_out_without_heat():
    sim = auto(gravity=(0., -9.81, 0.))
    with pytest.raises(RuntimeError, match="baking was not started"):
        sim.Advance(20)
    assert sim.IsSettling and sim.settling_reason == "timeout" and sim.baking_time == 0
    np.testing.assert_allclose(to_np(sim.current_state.transport_state.temperatures), 293.15, atol=1e-12)


@pytest.mark.gpu
def test_brief_quiet_and_deformation_cannot_trigger_transition():
    import torch
    from baking_b200 import arrays
    from baking_b200.physics.quasistatic import SettlingMetrics
    sim = auto()
    sim.Advance(3)
    assert sim.settling_quiet_steps == 1
    assign(sim.current_state.particle_velocities, np.tile([.01, 0., 0.], (sim.particle_data.particle_count, 1)))
    sim.Step()
    assert sim.IsSettling and sim.settling_quiet_steps == 0
    old = arrays.from_numpy(np.eye(3, dtype=np.float32)[None], "f4")
    changed = arrays.from_numpy((np.eye(3, dtype=np.float32) * 1.01)[None], "f4")
    metrics = torch.zeros(3, device="cuda")
    SettlingMetrics(arrays.vec3s(1), arrays.from_numpy((np.eye(3, dtype=np.float32) * .1)[None], "f4"), old, changed,
                    metrics, .01)
    values = metrics.cpu().numpy()
    assert values[0] == 0 and values[1] > .1 and values[2] > .9
