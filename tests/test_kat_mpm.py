"""Known answers of the reference's mechanics tests, on the oracle and on the device.

Restates tests/test_mpm.py:18-73, tests/test_elastic_material.py:10-39 and
tests/test_mesh_reconstruction.py:15-102 of the reference.
"""
import numpy as np
import pytest

from baking_b200.config import MaterialConfig, SimulationConfig
from baking_b200.geometry import CreateDemoMesh, SampleParticles, ValidateTetMesh
from tests.kat_api import ENGINES, Api
from tests.scenes import assign, to_np


def build(api, gravity=(0.0, 0.0, 0.0), initial_velocity=(0.2, -0.1, 0.05), time_step=1e-4):
    mesh = CreateDemoMesh(3)
    return api.simulator(mesh, SampleParticles(mesh, 1000.0, 4), api.sim_config(gravity=gravity, time_step=time_step),
                         MaterialConfig(), initial_velocity)


@pytest.mark.parametrize("engine", ENGINES)
def test_free_translation_conserves_mass_momentum_and_shape(engine):
    sim = build(Api(engine))
    x0 = to_np(sim.current_state.particle_positions).copy()
    v0_vertices = to_np(sim.vertex_positions).copy()
    velocity = np.array(sim.initial_velocity)
    mass0 = to_np(sim.particle_data.particle_masses).sum(dtype=np.float64)
    stats = sim.Advance(30)
    t = 30 * sim.simulation_config.time_step
    st = sim.current_state
    np.testing.assert_allclose(to_np(st.particle_positions), x0 + t * velocity, atol=2e-6)
    np.testing.assert_allclose(to_np(st.particle_velocities), np.tile(velocity, (len(x0), 1)), atol=2e-5)
    np.testing.assert_allclose(to_np(st.deformation_gradients), np.tile(np.eye(3), (len(x0), 1, 1)), atol=1e-5)
    np.testing.assert_allclose(to_np(sim.vertex_positions), v0_vertices + t * velocity, atol=2e-6)
    np.testing.assert_allclose(stats["grid_mass"], mass0, rtol=1e-6)
    assert stats["unmapped_mesh_vertices"] == 0


@pytest.mark.parametrize("engine", ENGINES)
def test_free_fall_matches_symplectic_euler(engine):
    sim = build(Api(engine), gravity=(0.0, -9.81, 0.0), initial_velocity=(0.0, 0.0, 0.0))
    x0 = to_np(sim.current_state.particle_positions).copy()
    steps, dt = 40, sim.simulation_config.time_step
    sim.Advance(steps)
    expected = x0.copy()
    expected[:, 1] -= 9.81 * dt ** 2 * steps * (steps + 1) / 2
    v = np.zeros_like(x0)
    v[:, 1] = -9.81 * dt * steps
    np.testing.assert_allclose(to_np(sim.current_state.particle_positions), expected, atol=1.5e-6)
    np.testing.assert_allclose(to_np(sim.current_state.particle_velocities), v, atol=1e-5)


@pytest.mark.gpu
def test_reset_and_snapshot(tmp_path):
    sim = build(Api("cuda"))
    x0 = to_np(sim.current_state.particle_positions).copy()
    sim.Advance(5)
    path = tmp_path / "snapshot.npz"
    sim.SaveSnapshot(path)
    with np.load(path) as data:
        np.testing.assert_allclose(data["particle_positions"], to_np(sim.current_state.particle_positions))
        assert data["simulation_time"] == 5 * sim.simulation_config.time_step
    sim.Reset()
    assert sim.step_count == 0
    np.testing.assert_array_equal(to_np(sim.current_state.particle_positions), x0)


def test_excessive_time_step_rejected():
    from dataclasses import replace
    with pytest.raises(ValueError, match="CFL"):
        replace(SimulationConfig(), time_step=1.0).Validate(MaterialConfig())


@pytest.mark.parametrize("engine", ENGINES)
def test_elastic_reference_rotation_and_stretch(engine):
    api = Api(engine)
    mesh = CreateDemoMesh(1)
    mc = MaterialConfig()
    sim = api.simulator(mesh, SampleParticles(mesh, 1000.0, 1), api.sim_config(), mc)
    F = np.tile(np.eye(3, dtype=np.float32), (6, 1, 1))
    a = 0.4
    F[1] = [[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]]
    F[2] = np.diag([1.1, 1.0, 1.0])
    F[3] = np.diag([0.9, 1.0, 1.0])
    assign(sim.current_state.deformation_gradients, F)
    sim.material.ComputeStress(sim.current_state, sim.kirchhoff_stresses, sim.error_flags)
    tau = to_np(sim.kirchhoff_stresses)
    expected = [mc.shear_modulus * (f @ f.T - np.eye(3)) + mc.lame_lambda * np.log(np.linalg.det(f)) * np.eye(3)
                for f in F]
    np.testing.assert_allclose(tau, expected, rtol=1e-5, atol=0.005)
    np.testing.assert_allclose(tau[:2], 0.0, atol=0.005)
    assert tau[2, 0, 0] > 0.0 and tau[3, 0, 0] < 0.0
    F[0, 0, 0] = -1.0
    assign(sim.current_state.deformation_gradients, F)
    sim.material.ComputeStress(sim.current_state, sim.kirchhoff_stresses, sim.error_flags)
    assert to_np(sim.error_flags)[0] == 1


def _reconstruct(api, mesh, samples, x, F):
    n = len(x)
    if api.engine == "oracle":
        from oracle import ora
        from baking_b200.geometry import MeshBindingTables_build
        t = MeshBindingTables_build(mesh, samples)
        out = ora.f32(len(mesh.vertex_positions), 3)
        ora.reconstruct_mesh_vertices(np.ascontiguousarray(x, np.float32), np.ascontiguousarray(F, np.float32),
                                      np.ascontiguousarray(mesh.vertex_positions, np.float32), t.binding_offsets,
                                      t.binding_particles, np.ascontiguousarray(t.binding_weights, np.float32),
                                      np.ascontiguousarray(t.reference_offsets, np.float32), out)
        return out, t.unmapped_vertex_count
    from baking_b200 import arrays
    from baking_b200.geometry.mesh_tracking import ParticleMeshBinding
    from baking_b200.physics.state import AllocateState
    binding = ParticleMeshBinding(mesh, samples, api.device)
    st = AllocateState(n, api.device)
    assign(st.particle_positions, x)
    assign(st.deformation_gradients, F)
    out = arrays.vec3s(len(mesh.vertex_positions), device=api.device)
    binding.Reconstruct(st, out)
    return to_np(out), binding.unmapped_vertex_count


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("count", [1, 4, 7])
def test_reconstruction_reproduces_affine_deformation(engine, count):
    api = Api(engine)
    mesh = CreateDemoMesh(2)
    samples = SampleParticles(mesh, 1000.0, count)
    a = 0.7
    R = np.array([[np.cos(a), -np.sin(a), 0.0], [np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
    shift = np.array([0.15, -0.1, 0.05])
    for A in (np.eye(3), R, R @ np.array([[1.2, 0.2, 0.0], [0.0, 0.8, 0.1], [0.0, 0.0, 1.1]])):
        x = (samples.particle_positions @ A.T + shift).astype(np.float32)
        F = np.tile(A.astype(np.float32), (len(x), 1, 1))
        out, _ = _reconstruct(api, mesh, samples, x, F)
        np.testing.assert_allclose(out, mesh.vertex_positions @ A.T + shift, rtol=1e-6, atol=4e-7)


@pytest.mark.parametrize("engine", ENGINES)
def test_shared_vertices_blend_incident_particle_predictions(engine):
    api = Api(engine)
    mesh = ValidateTetMesh(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -2], [5, 5, 5]], float),
                           np.array([[0, 1, 2, 3], [0, 2, 1, 4]]))
    samples = SampleParticles(mesh, 1000.0, 1)
    x = samples.particle_positions.copy()
    x[0] += [0.1, 0.0, 0.0]
    x[1] += [0.0, 0.2, 0.0]
    F = np.array([np.diag([1.1, 0.9, 1.0]), np.diag([0.8, 1.2, 1.0])])
    out, unmapped = _reconstruct(api, mesh, samples, x.astype(np.float32), F.astype(np.float32))
    expected = mesh.vertex_positions.copy()
    for v in range(len(expected)):
        incident = [p for p, t in enumerate(samples.source_tets) if v in mesh.tet_indices[t]]
        if incident:
            preds = [x[p] + F[p] @ (mesh.vertex_positions[v] - samples.particle_positions[p]) for p in incident]
            expected[v] = np.average(preds, axis=0, weights=samples.reference_volumes[incident])
    np.testing.assert_allclose(out, expected, atol=3e-7)
    assert unmapped == 1
    np.testing.assert_array_equal(out[5], mesh.vertex_positions[5].astype(np.float32))


@pytest.mark.gpu
def test_mesh_updates_after_substeps_and_snapshot(tmp_path):
    api = Api("cuda")
    mesh = CreateDemoMesh(2)
    velocity = np.array([0.2, 0.1, -0.05])
    sim = api.simulator(mesh, SampleParticles(mesh, 1000.0, 4), api.sim_config(gravity=(0.0, 0.0, 0.0)),
                        MaterialConfig(), velocity)
    dt = sim.simulation_config.time_step
    for _ in range(3):
        sim.Advance(5)
        np.testing.assert_allclose(to_np(sim.vertex_positions), mesh.vertex_positions + sim.step_count * dt * velocity,
                                   atol=2e-6)
        assert sim.mesh_step_count == sim.step_count
    sim.Step()
    sim.SaveSnapshot(tmp_path / "mesh.npz")
    with np.load(tmp_path / "mesh.npz") as data:
        np.testing.assert_allclose(data["vertices"], mesh.vertex_positions + sim.step_count * dt * velocity, atol=2e-6)
        np.testing.assert_array_equal(data["tetrahedra"], mesh.tet_indices)
    sim.Reset()
    np.testing.assert_array_equal(to_np(sim.vertex_positions), mesh.vertex_positions.astype(np.float32))
    assert sim.mesh_step_count == 0
