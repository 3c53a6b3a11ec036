"""Known answers of the reference's transport and gas tests, on the oracle and on the device.

Restates tests/test_transport.py:30-213 and tests/test_gas.py:259-436 of the reference
(gradient tests are restated with the adjoint; recorder checks are out of scope).
"""
from dataclasses import replace

import numpy as np
import pytest

from baking_b200.config import DingConfig, MaterialConfig, TransportConfig
from baking_b200.geometry import BoundaryFaces, CreateDemoMesh, SampleParticles
from tests.kat_api import ENGINES, Api
from tests.scenes import assign, build_gas, build_transport, to_np

GAS_CONSTANT = 8.31446261815324


def thermal_steps(sim, count, dt):
    # Geometry frozen to isolate transport (reference tests/test_transport.py:23-27).
    for _ in range(count):
        sim.current_state = sim.transport.Advance(sim.current_state, dt)
    return sim.current_state.transport_state


@pytest.mark.parametrize("engine", ENGINES)
def test_insulated_uniform_temperature_and_water_conservation(engine):
    config = TransportConfig(enabled=True, heat_transfer=0., tray_heat_transfer=0., surface_water_loss=0.)
    sim = build_transport(engine, config)
    water0 = to_np(sim.current_state.transport_state.water_masses).sum()
    result = thermal_steps(sim, 8, 0.001)
    np.testing.assert_allclose(to_np(result.temperatures), config.initial_temperature_k, atol=1e-12)
    np.testing.assert_allclose(to_np(result.water_masses).sum(), water0, rtol=2e-7)
    masses = to_np(result.water_masses).copy()
    x = to_np(sim.current_state.particle_positions)
    masses *= np.where(x[:, 0] < 0.5, 1.5, 0.5)
    assign(result.water_masses, masses)
    after = to_np(thermal_steps(sim, 8, 0.01).water_masses)
    np.testing.assert_allclose(after.sum(), masses.sum(), rtol=2e-7)
    assert (after[masses > masses.mean()] - masses[masses > masses.mean()]).sum() < 0


@pytest.mark.parametrize("engine", ENGINES)
def test_boundary_area_tray_and_water_stress(engine):
    api = Api(engine)
    sim = build_transport(engine)
    faces, owners = BoundaryFaces(sim.tet_mesh, sim.particle_samples)
    assert len(faces) == 48
    n = sim.particle_data.particle_count
    vertices = np.ascontiguousarray(sim.tet_mesh.vertex_positions, np.float32)
    if engine == "oracle":
        from oracle import ora
        exposed, contact = ora.f64(n), ora.f64(n)
        ora.surface_areas(vertices, faces, owners, exposed, contact, .45, .001)
        before, after = ora.f32(n, 3, 3), ora.f32(n, 3, 3)
        ora.water_stress(sim.current_state.deformation_gradients, np.full(n, .3), before, after, .4, 10000.)
    else:
        import torch
        from baking_b200 import arrays
        from baking_b200.physics.thermal_water import SurfaceAreas, WaterStress
        exposed = torch.zeros(n, dtype=torch.float64, device=api.device)
        contact = torch.zeros(n, dtype=torch.float64, device=api.device)
        SurfaceAreas(arrays.from_numpy(vertices, "f4", api.device), torch.as_tensor(faces, device=api.device),
                     torch.as_tensor(owners, device=api.device), exposed, contact, .45, .001)
        before = arrays.mat33s(n, device=api.device)
        after = arrays.mat33s(n, device=api.device)
        WaterStress(sim.current_state.deformation_gradients, torch.full((n,), .3, dtype=torch.float64,
                                                                        device=api.device), before, after, .4, 10000.)
    np.testing.assert_allclose(to_np(exposed).sum(), .45, rtol=2e-6)
    np.testing.assert_allclose(to_np(contact).sum(), .09, rtol=2e-6)
    np.testing.assert_allclose(to_np(after), np.tile(np.eye(3) * 1000, (n, 1, 1)), rtol=1e-6)


@pytest.mark.parametrize("engine", ENGINES)
def test_outside_in_water_loss_heat_balance_and_latent_cooling(engine):
    common = TransportConfig(enabled=True, conductivity=20., specific_heat=100., heat_transfer=2000.,
                             surface_water_loss=1e-5, water_diffusivity=1e-8, water_stress=0.)
    means = []
    for latent in (0., 2.26e6):
        sim = build_transport(engine, replace(common, latent_heat=latent), subdivisions=3)
        state = thermal_steps(sim, 40, .001)
        t = to_np(state.temperatures)
        p = sim.particle_samples.particle_positions
        surface = np.zeros(len(t), bool)
        surface[to_np(sim.transport.owners)] = True
        core = np.linalg.norm(p - np.array([.5, .6, .5]), axis=1) < .07
        assert t[surface].mean() > t[core].mean()
        initial_water = common.water_density * common.initial_saturation * .027
        assert to_np(state.water_masses).sum() < initial_water
        np.testing.assert_allclose(to_np(state.water_masses).sum() + to_np(state.water_losses).sum(), initial_water,
                                   rtol=2e-7)
        np.testing.assert_allclose(np.dot(to_np(sim.transport.capacities), t - common.initial_temperature_k),
                                   to_np(state.heat_exchanges).sum(), rtol=2e-6)
        means.append(t.mean())
    assert means[1] < means[0]


@pytest.mark.parametrize("engine", ENGINES)
def test_local_temperature_changes_gas_and_plastic_parameters(engine):
    config = TransportConfig(enabled=True, conductivity=0., heat_transfer=0., tray_heat_transfer=0.,
                             water_diffusivity=0., surface_water_loss=0., water_stress=0.)
    sim = build_transport(engine, config, gas=True)
    n = sim.particle_data.particle_count
    values = np.linspace(300., 360., n)
    assign(sim.current_state.transport_state.temperatures, values)
    before = to_np(sim.current_state.material_state.gas_moles).copy()
    dt = sim.simulation_config.time_step
    sim.Step()
    internal = sim.current_state.material_state
    ding = sim.material.ding_config
    expected = before + dt * 1000 * ding.gas_production_rate * np.exp(
        -((values - ding.gas_reaction_temperature_k) / ding.gas_reaction_width_k) ** 2)
    np.testing.assert_allclose(to_np(internal.gas_moles) - before, expected - before, rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(to_np(internal.temperatures), values, atol=2e-5)
    knots, factors = ding.temperature_knots_k, ding.yield_factors
    np.testing.assert_allclose(to_np(internal.yield_stresses),
                               [ding.yield_stress * float(np.interp(t, knots, factors)) for t in values], rtol=1e-5)
    np.testing.assert_array_equal(to_np(internal.gelled), values >= knots[-1])
    J = np.linalg.det(to_np(sim.current_state.deformation_gradients))
    pressure = expected * GAS_CONSTANT * to_np(internal.temperatures) / (J * to_np(internal.porosities))
    np.testing.assert_allclose(to_np(internal.gas_pressures), pressure, rtol=5e-7)


@pytest.mark.parametrize("engine", ENGINES)
def test_water_disabled_keeps_water_and_is_deterministic(engine):
    config = TransportConfig(enabled=True, water_enabled=False)
    a, b = build_transport(engine, config), build_transport(engine, config)
    water0 = to_np(a.current_state.transport_state.water_masses).copy()
    for _ in range(3):
        a.Step()
        b.Step()
    np.testing.assert_allclose(to_np(a.current_state.particle_positions), to_np(b.current_state.particle_positions),
                               rtol=0, atol=1e-7)
    np.testing.assert_array_equal(to_np(a.current_state.transport_state.water_masses), water0)


@pytest.mark.parametrize("engine", ENGINES)
def test_explicit_transport_bound(engine):
    sim = build_transport(engine, TransportConfig(enabled=True, conductivity=1e8))
    with pytest.raises(RuntimeError, match="stability bound"):
        sim.transport.Advance(sim.current_state, .1)


def grid_decay(api, resolution, dt):
    # Insulated cosine heat mode T = 300 + 10 cos(pi x) exp(-D pi^2 t) (reference test_transport.py:181-202).
    n = resolution ** 3
    h = 1. / resolution
    coords = np.indices((resolution,) * 3)[0].reshape(-1)
    initial = 300 + 10 * np.cos(np.pi * (coords + .5) * h)
    T = api.array(initial, "f8")
    vol, cap = api.array(np.full(n, h ** 3), "f8"), api.array(np.full(n, 1000 * h ** 3), "f8")
    zero = api.zeros(n, "f8")
    dT, dW = api.zeros(n, "f8"), api.zeros(n, "f8")
    flags = api.zeros(2, "i4")
    for _ in range(round(.2 / dt)):
        api.diffuse_grid(vol, cap, T, zero, zero, zero, zero, zero, dT, dW, flags, 10., 0., 1000., 0, h, resolution,
                         dt)
        T += dT
    exact = 300 + (initial - 300) * np.exp(-.01 * np.pi ** 2 * .2)
    assert to_np(flags).max() == 0
    t = to_np(T)
    amplitude = np.dot(t - 300, initial - 300) / np.dot(initial - 300, initial - 300)
    return float(np.sqrt(np.mean((t - exact) ** 2))), float(amplitude)


@pytest.mark.parametrize("engine", ENGINES)
def test_grid_and_time_convergence(engine):
    api = Api(engine)
    errors = [grid_decay(api, n, .0005)[0] for n in (8, 16, 32)]
    assert errors[1] < .35 * errors[0] and errors[2] < .35 * errors[1]
    n = 16
    rate = 4 * .01 * n * n * np.sin(np.pi / (2 * n)) ** 2
    exact = np.exp(-rate * .2)
    time_errors = [abs(grid_decay(api, n, dt)[1] - exact) for dt in (.02, .01, .005)]
    assert time_errors[1] < .51 * time_errors[0] and time_errors[2] < .51 * time_errors[1]


# ------------------------------------------------------------------------ gas
@pytest.mark.parametrize("engine", ENGINES)
def test_ideal_gas_units_and_scaling(engine):
    moles, T = np.full(4, 0.2), np.array([300., 600., 300., 300.], np.float32)
    J, n = np.array([1., 1., 2., 1.], np.float32), np.array([.2, .2, .2, .1], np.float32)
    if engine == "oracle":
        from oracle import ora
        pressures = np.array([ora.gas_pressure(*map(float, args)) for args in zip(moles, T, J, n)])
    else:
        # The device formula through RefreshGas: moles R T / (J n) with F = J^(1/3) I.
        import torch
        from baking_b200 import arrays
        from baking_b200.physics.materials.gas import RefreshGas
        F = arrays.from_numpy(np.stack([np.eye(3) * np.float32(j) ** (1 / 3) for j in J]).astype(np.float32), "f4")
        out_moles = torch.zeros(4, dtype=torch.float64, device="cuda")
        p = torch.zeros(4, dtype=torch.float64, device="cuda")
        RefreshGas(torch.as_tensor(moles, device="cuda"), out_moles, F, torch.as_tensor(n, device="cuda"), p,
                   torch.as_tensor(T, device="cuda"))
        pressures = p.cpu().numpy()
    np.testing.assert_allclose(pressures / (GAS_CONSTANT * 300), [1, 2, 0.5, 2], rtol=2e-7)


@pytest.mark.parametrize("engine", ENGINES)
def test_stress_conversion_ambient_and_no_source_conservation(engine):
    api = Api(engine)
    material = api.ding_material(MaterialConfig(), DingConfig(gas_enabled=True, porosity=0.2, gas_production_rate=0.0))
    state = api.point(material)
    stress = api.zeros((1, 3, 3), "f4")
    flags = api.zeros(2, "i4")
    material.ComputeStress(state, stress, flags)
    np.testing.assert_allclose(to_np(stress), 0, atol=0.02)
    assign(state.material_state.gas_moles, to_np(state.material_state.gas_moles) * 2)
    material.ComputeStress(state, stress, flags)
    np.testing.assert_allclose(to_np(stress)[0], -101325 * np.eye(3), rtol=2e-6, atol=0.03)
    assign(state.deformation_gradients, (np.eye(3, dtype=np.float32) * np.float32(2 ** (1 / 3)))[None])
    material.ding_config = replace(material.ding_config, gas_ambient_pressure_pa=0)
    material.ComputeStress(state, stress, flags)
    np.testing.assert_allclose(to_np(stress)[0], -202650 * np.eye(3), rtol=2e-6, atol=0.05)
    assign(state.deformation_gradients, np.eye(3, dtype=np.float32)[None])
    moles0 = to_np(state.material_state.gas_moles).copy()
    for _ in range(10):
        state = api.point_step(material, state, np.eye(3), 0.01)
    np.testing.assert_array_equal(to_np(state.material_state.gas_moles), moles0)


@pytest.mark.parametrize("engine", ENGINES)
def test_local_gaussian_source_constant_temperature(engine):
    api = Api(engine)
    for steps in (1, 20, 100):
        T = api.array([333.15], "f8")
        old = api.zeros(1, "f8")
        pressure = api.zeros(1, "f8")
        F = api.array(np.eye(3, dtype=np.float32)[None], "f4")
        porosity = api.array([.2], "f4")
        parameter = api.array([.002], "f4")
        for _ in range(steps):
            out = api.zeros(1, "f8")
            if engine == "oracle":
                from oracle import ora
                ora.local_gas(old, T, T, out, pressure, F, porosity, parameter, 1000., 333.15, 15., .1 / steps, 1)
            else:
                from baking_b200.physics.thermal_water import LocalGas
                LocalGas(old, T, T, out, pressure, F, porosity, parameter, 1000., 333.15, 15., .1 / steps, 1)
            old = out
        np.testing.assert_allclose(to_np(old), .2, rtol=2e-6)


@pytest.mark.parametrize("engine", ENGINES)
def test_coupled_compaction_consistency_and_small_pores(engine):
    api = Api(engine)
    material = api.ding_material(MaterialConfig(), DingConfig(gas_enabled=True, porosity=0.2, yield_stress=100,
                                                              viscosity=1e8, gas_production_rate=0))
    state = api.point(material)
    for k in range(30):
        state = api.point_step(material, state, np.eye(3) * (1 - 0.001 * (k + 1)), 0.001)
        internal = state.material_state
        n = to_np(internal.porosities)[0]
        assert 0 < n <= 0.200001
        np.testing.assert_allclose(to_np(internal.porosities), np.linalg.det(to_np(internal.plastic_gradients)) - 1 + 0.2,
                                   atol=2e-6)
        assert to_np(internal.porosity_residuals)[0] < 1e-6
    assert n < 0.199
    material = api.ding_material(MaterialConfig(), DingConfig(gas_enabled=True, porosity=1e-7, gas_production_rate=0))
    state = api.point(material)
    stress = api.zeros((1, 3, 3), "f4")
    material.ComputeStress(state, stress, api.zeros(2, "i4"))
    assert np.isfinite(to_np(stress)).all()
    assign(state.material_state.gas_moles, np.array([101325 * 0.2 / (GAS_CONSTANT * 293.15)]))
    material.ComputeStress(state, stress, api.zeros(2, "i4"))
    assert np.isfinite(to_np(stress)).all()
    assert abs(to_np(stress)[0, 0, 0]) > 1e10
    from baking_b200.config import SimulationConfig
    material.simulation_config = SimulationConfig()
    with pytest.raises(RuntimeError, match="Gas acoustic CFL"):
        material.ComputeStress(state, stress, api.zeros(2, "i4"))
    with pytest.raises(ValueError, match="positive initial porosity"):
        DingConfig(gas_enabled=True, porosity=0).Validate()


@pytest.mark.parametrize("engine", ENGINES)
def test_gas_expansion_and_source_effect(engine):
    volumes = []
    for rate in (0.0, 0.005):
        sim = build_gas(engine, rate=rate)
        sim.Advance(100)
        volumes.append(float(np.linalg.det(to_np(sim.current_state.deformation_gradients)).mean()))
    assert volumes[1] > volumes[0] + 0.001
    sim.Reset()
    np.testing.assert_allclose(to_np(sim.current_state.material_state.gas_moles), 1000 * 0.2 / (GAS_CONSTANT * 333.15))


@pytest.mark.parametrize("engine", ENGINES)
def test_gas_time_step_sensitivity(engine):
    results = []
    for dt in (0.0005, 0.00025):
        sim = build_gas(engine, dt=dt)
        sim.Advance(round(0.05 / dt))
        results.append(float(np.linalg.det(to_np(sim.current_state.deformation_gradients)).mean()))
    np.testing.assert_allclose(results[0], results[1], rtol=0.003)


@pytest.mark.parametrize("engine", ENGINES)
def test_near_closure_consistent_return_does_not_overshoot(engine):
    n0, start = 0.2, 3.725290298461914e-7
    volume = 1.0 - n0 + start
    args = (4.115, 29.464, 0.001052, 0.003390, -0.0230067)
    if engine == "oracle":
        from oracle import ora
        n = ora.solve_porosity(*args, volume, n0)
        pred = ora.porosity_prediction(float(np.float32(n)), *args, volume, n0)
    else:
        from baking_b200.physics.materials.porous_return import SolvePorosity
        out, prediction = SolvePorosity(*[[a] for a in args], [volume], n0)
        n, pred = float(out[0]), float(prediction[0])
    assert 0 < n < start
    np.testing.assert_allclose(n, pred, atol=1e-12)
