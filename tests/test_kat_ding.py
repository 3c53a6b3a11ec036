"""Known answers of the reference's Ding material tests, on the oracle and on the device.

Restates tests/test_ding.py:32-205 and tests/test_ding_thermal.py:246-439 of the reference
(the gradient tests are restated with the adjoint).
"""
from dataclasses import replace

import numpy as np
import pytest

from baking_b200.config import DingConfig, MaterialConfig, TransportConfig
from baking_b200.geometry import CreateDemoMesh, SampleParticles
from tests.kat_api import ENGINES, Api
from tests.scenes import assign, to_np

ms = lambda s, name: to_np(getattr(s.material_state, name))  # noqa: E731


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("stretch", [1.25, 0.8])
def test_point_load_hold_unload(engine, stretch):
    api = Api(engine)
    material = api.ding_material(MaterialConfig(), DingConfig(yield_stress=500.0, viscosity=1e10))
    state = api.point(material)
    F = np.diag([stretch, 1.0, 1.0])
    state = api.point_step(material, state, F)
    initial = ms(state, "kirchhoff_stresses")[0].copy()
    energies = []
    mu, lam = material.material_config.shear_modulus, material.material_config.lame_lambda
    for _ in range(40):
        state = api.point_step(material, state, F)
        e = np.log(np.linalg.svd(ms(state, "elastic_gradients")[0], compute_uv=False))
        energies.append(mu * np.dot(e, e) + 0.5 * lam * e.sum() ** 2)
    final = ms(state, "kirchhoff_stresses")[0]
    dev = lambda t: t - np.eye(3) * np.trace(t) / 3  # noqa: E731
    assert initial[0, 0] * (stretch - 1) > 0
    assert np.linalg.norm(dev(final)) < np.linalg.norm(dev(initial))
    assert np.max(np.diff(energies)) < 0.01
    Fp = ms(state, "plastic_gradients")[0]
    np.testing.assert_allclose(np.linalg.det(Fp), 1.0, atol=2e-5)
    np.testing.assert_allclose(ms(state, "elastic_gradients")[0] @ Fp, F, atol=1e-5)
    assert ms(state, "return_residuals").max() < 1e-5
    residual_gradient = Fp.copy()
    state = api.point_step(material, state, residual_gradient)
    np.testing.assert_allclose(ms(state, "kirchhoff_stresses"), 0, atol=0.5)
    assert np.linalg.norm(residual_gradient - np.eye(3)) > 0.01


@pytest.mark.parametrize("engine", ENGINES)
def test_elastic_limit_objectivity_and_porosity(engine):
    api = Api(engine)
    material = api.ding_material(MaterialConfig(), DingConfig(yield_stress=1e9))
    state = api.point(material)
    F = np.diag([1.1, 0.95, 1.02])
    state = api.point_step(material, state, F)
    e = np.log(np.diag(F))
    mu, lam = material.material_config.shear_modulus, material.material_config.lame_lambda
    expected = np.diag(2 * mu * e + lam * e.sum())
    np.testing.assert_allclose(ms(state, "kirchhoff_stresses")[0], expected, rtol=2e-5, atol=0.02)
    np.testing.assert_allclose(ms(state, "plastic_gradients")[0], np.eye(3), atol=1e-6)
    a = 0.5
    R = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    state = api.point_step(material, state, R @ F)
    np.testing.assert_allclose(ms(state, "kirchhoff_stresses")[0], R @ expected @ R.T, atol=0.05)
    for porosity in (0.0, 0.2):
        material = api.ding_material(MaterialConfig(), DingConfig(yield_stress=100.0, porosity=porosity))
        state = api.point_step(material, api.point(material), np.eye(3) * 0.9)
        volume = np.linalg.det(ms(state, "plastic_gradients")[0])
        if porosity == 0:
            np.testing.assert_allclose(volume, 1, atol=1e-5)
        else:
            assert volume < 0.999


@pytest.mark.parametrize("engine", ENGINES)
def test_mpm_and_internal_snapshots(engine):
    api = Api(engine)
    mesh = CreateDemoMesh(2)
    sim = api.simulator(mesh, SampleParticles(mesh, 1000.0, 4), api.sim_config(), MaterialConfig(model="ding2019"),
                        ding_config=DingConfig(yield_stress=100.0, viscosity=1e8))
    x = to_np(sim.current_state.particle_positions).copy()
    rates = np.diag([1.5, -0.75, 0.2]).astype(np.float32)
    assign(sim.current_state.particle_velocities, (x - np.array([0.5, 0.6, 0.5], np.float32)) @ rates.T)
    assign(sim.current_state.affine_velocities, np.tile(rates, (len(x), 1, 1)))
    sim.Advance(600)
    s = sim.current_state
    assert np.max(np.abs(ms(s, "plastic_gradients") - np.eye(3))) > 1e-4
    np.testing.assert_allclose(ms(s, "elastic_gradients") @ ms(s, "plastic_gradients"),
                               to_np(s.deformation_gradients), atol=2e-5)
    sim.Reset()
    np.testing.assert_allclose(ms(sim.current_state, "elastic_gradients"), np.tile(np.eye(3), (len(x), 1, 1)))


@pytest.mark.parametrize("engine", ENGINES)
def test_local_stationarity_and_viscosity_dependence(engine):
    api = Api(engine)
    norms = []
    for eta in (1e9, 1e11):
        material = api.ding_material(MaterialConfig(), DingConfig(yield_stress=300.0, viscosity=eta, porosity=0.2))
        F = np.diag([1.2, 0.9, 1.04])
        state = api.point_step(material, api.point(material), F)
        tau = np.diag(ms(state, "kirchhoff_stresses")[0]).astype(float)
        mu, lam = material.material_config.shear_modulus, material.material_config.lame_lambda
        stiffness = 2 * mu * np.eye(3) + lam * np.ones((3, 3))
        trial = stiffness @ np.log(np.diag(F))
        mean = tau.mean()
        dev = tau - mean
        a = material.pressure_coefficient
        f = 1.5 * np.dot(dev, dev) + a * mean ** 2 - 300.0 ** 2
        grad_f = 3 * dev + (2 * a / 3) * mean * np.ones(3)
        stationarity = np.linalg.inv(stiffness) @ (tau - trial) + 0.01 / eta * max(f, 0) * grad_f
        np.testing.assert_allclose(stationarity, 0, atol=2e-6)
        norms.append(np.linalg.norm(dev))
    assert norms[1] > norms[0]


@pytest.mark.parametrize("engine", ENGINES)
def test_load_rate_dependence(engine):
    api = Api(engine)
    stresses = []
    for total in (0.02, 0.2):
        material = api.ding_material(MaterialConfig(), DingConfig(yield_stress=500.0, viscosity=1e10))
        state = api.point(material)
        for k in range(20):
            s = np.exp(np.log(1.2) * (k + 1) / 20)
            state = api.point_step(material, state, np.diag([s, 1.0, 1.0]), total / 20)
        tau = ms(state, "kirchhoff_stresses")[0]
        stresses.append(np.linalg.norm(tau - np.trace(tau) / 3 * np.eye(3)))
    assert stresses[0] > stresses[1]


# ---------------------------------------------------------------- thermal Ding
SETTING = DingConfig(temperature_enabled=True, yield_stress=500.0, viscosity=1e9,
                     temperature_knots_k=(278.15, 293.15, 328.15, 353.15),
                     yield_factors=(1.5, 1.0, 0.5, 3.0), viscosity_factors=(1.5, 1.0, 0.5, 5.0))


@pytest.mark.parametrize("engine", ENGINES)
def test_rising_penalty_viscosity_during_setting(engine):
    api = Api(engine)
    SETTING.Validate()
    for T, factor in ((328.15, 0.5), (340.65, 2.75), (353.15, 5.0)):
        material = api.ding_material(MaterialConfig(), SETTING, initial_temperature_k=T)
        state = api.point(material)
        for checked in (state, api.point_step(material, state, np.eye(3))):
            np.testing.assert_allclose(ms(checked, "viscosities"), SETTING.viscosity * factor, rtol=2e-6)
    norms = []
    for hot in (0.5, 5.0):
        config = replace(SETTING, viscosity_factors=(1.5, 1.0, 0.5, hot))
        material = api.ding_material(MaterialConfig(), config, initial_temperature_k=353.15)
        state = api.point_step(material, api.point(material), np.diag([1.2, 0.9, 1.04]))
        assert np.isfinite(ms(state, "kirchhoff_stresses")).all()
        norms.append(np.linalg.norm(ms(state, "kirchhoff_stresses")))
    assert norms[1] > norms[0]


@pytest.mark.parametrize("engine", ENGINES)
def test_temperature_and_porosity_parameter_values(engine):
    api = Api(engine)
    config = DingConfig(temperature_enabled=True)
    for T, yf, vf in ((260.0, 1.5, 1.5), (278.15, 1.5, 1.5), (293.15, 1.0, 1.0), (303.15, 0.6, 0.6),
                      (313.15, 0.2, 0.2), (333.15, 1.1, 0.125), (353.15, 2.0, 0.05), (400.0, 2.0, 0.05)):
        material = api.ding_material(MaterialConfig(), config, initial_temperature_k=T)
        state = api.point(material)
        for checked in (state, api.point_step(material, state, np.eye(3))):
            np.testing.assert_allclose(ms(checked, "yield_stresses"), config.yield_stress * yf, rtol=2e-6)
            np.testing.assert_allclose(ms(checked, "viscosities"), config.viscosity * vf, rtol=2e-6)
            np.testing.assert_allclose(ms(checked, "temperatures"), T, atol=2e-5)
    porosities = np.array([0.0, 0.01, 0.1, 0.2, 0.5, 0.999], dtype=np.float32)
    if engine == "oracle":
        from oracle import ora
        coefficients = np.array([ora.porosity_coefficient(float(p)) for p in porosities])
    else:
        from baking_b200.physics.materials.porous_return import PorosityCoefficients
        coefficients = PorosityCoefficients(porosities).cpu().numpy()
    expected = [0.0] + [9 / (4 * np.log(1 / p) ** 2 * (3.5 * p + 1)) for p in porosities[1:]]
    np.testing.assert_allclose(coefficients, expected, rtol=5e-5)
    assert np.all(np.diff(coefficients) > 0)


@pytest.mark.parametrize("engine", ENGINES)
def test_initial_porosity_and_elastic_versus_plastic_volume(engine):
    api = Api(engine)
    for porosity in (0.0, 0.2, 0.5):
        material = api.ding_material(MaterialConfig(), DingConfig(yield_stress=1e9, porosity=porosity))
        state = api.point(material)
        np.testing.assert_allclose(ms(state, "porosities"), porosity)
        state = api.point_step(material, state, np.diag([1.1, 0.95, 1.02]))
        np.testing.assert_allclose(ms(state, "porosities"), porosity, atol=1e-6)
    for stretch in (0.98, 1.02):
        material = api.ding_material(MaterialConfig(), DingConfig(yield_stress=100.0, porosity=0.2))
        state = api.point(material)
        for _ in range(5):
            state = api.point_step(material, state, np.eye(3) * stretch)
            volume = np.linalg.det(ms(state, "plastic_gradients"))
            np.testing.assert_allclose(ms(state, "porosities"), volume - 1 + 0.2, atol=2e-7)
        assert (ms(state, "porosities")[0] - 0.2) * (stretch - 1) > 0


@pytest.mark.parametrize("engine", ENGINES)
def test_updated_porosity_defines_next_return_map(engine):
    api = Api(engine)
    config = DingConfig(yield_stress=100.0, porosity=0.2)
    material = api.ding_material(MaterialConfig(), config)
    F = np.eye(3) * 0.98
    state = api.point_step(material, api.point(material), F)
    old_stress = ms(state, "kirchhoff_stresses")[0].copy()
    old_porosity = float(ms(state, "porosities")[0])
    state = api.point_step(material, state, F)
    tau = np.linalg.eigvalsh(ms(state, "kirchhoff_stresses")[0]).astype(float)
    trial = np.linalg.eigvalsh(old_stress).astype(float)
    mu, lam = material.material_config.shear_modulus, material.material_config.lame_lambda
    compliance = np.linalg.inv(2 * mu * np.eye(3) + lam * np.ones((3, 3)))
    a = 9 / (4 * np.log(1 / old_porosity) ** 2 * (3.5 * old_porosity + 1))
    mean = tau.mean()
    dev = tau - mean
    f = 1.5 * np.dot(dev, dev) + a * mean ** 2 - config.yield_stress ** 2
    grad_f = 3 * dev + (2 * a / 3) * mean
    residual = compliance @ (tau - trial) + 0.01 / config.viscosity * max(f, 0) * grad_f
    np.testing.assert_allclose(residual, 0, atol=2e-6)
    assert abs(old_porosity - config.porosity) > 1e-4


@pytest.mark.parametrize("engine", ENGINES)
def test_heating_changes_response_without_thermal_expansion(engine):
    api = Api(engine)
    norms = []
    for T in (293.15, 313.15, 353.15):
        config = DingConfig(temperature_enabled=True, yield_stress=500.0, porosity=0.2)
        material = api.ding_material(MaterialConfig(), config, initial_temperature_k=T)
        state = api.point(material)
        for _ in range(20):
            state = api.point_step(material, state, np.diag([1.05, 1 / np.sqrt(1.05), 1 / np.sqrt(1.05)]))
        tau = ms(state, "kirchhoff_stresses")[0]
        norms.append(float(np.linalg.norm(tau - np.trace(tau) / 3 * np.eye(3))))
    assert norms[1] < norms[0] < norms[2]
    material = api.ding_material(MaterialConfig(), DingConfig(temperature_enabled=True, porosity=0.2))
    state = api.point(material)
    for _ in range(100):
        state = api.point_step(material, state, np.eye(3), 0.025)
    np.testing.assert_allclose(ms(state, "elastic_gradients"), np.eye(3, dtype=np.float32)[None], atol=2e-6)
    np.testing.assert_allclose(ms(state, "kirchhoff_stresses"), 0.0, atol=0.05)
    np.testing.assert_allclose(ms(state, "porosities"), 0.2, atol=2e-6)


@pytest.mark.parametrize("values", [dict(temperature_knots_k=(278, 293, 290, 353)),
                                    dict(viscosity_factors=(1, float("inf"), 0.2, 0.1)),
                                    dict(viscosity_factors=(1, 0.5, 0.2, 0)), dict(yield_factors=(1, 2, 0.2, 3)),
                                    dict(porosity=-0.1), dict(porosity=1.0)])
def test_temperature_and_porosity_domains(values):
    with pytest.raises(ValueError):
        replace(DingConfig(), **values).Validate()


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("porosity,stretch", [(0.95, 1.2), (0.2, 0.7)])
def test_porosity_exceeding_domain_is_reported_without_clamping(engine, porosity, stretch):
    api = Api(engine)
    material = api.ding_material(MaterialConfig(), DingConfig(porosity=porosity, yield_stress=100.0, viscosity=1e4))
    with pytest.raises(RuntimeError, match="porosity left"):
        api.point_step(material, api.point(material), np.eye(3) * stretch)


def thermal_simulator(api, viscosity=1e8):
    mesh = CreateDemoMesh(1)
    sim = api.simulator(mesh, SampleParticles(mesh, 1000.0, 4), api.sim_config(time_step=1e-4, gravity=(0., 0., 0.)),
                        MaterialConfig(model="ding2019"),
                        ding_config=DingConfig(temperature_enabled=True, porosity=0.2, yield_stress=100.0,
                                               viscosity=viscosity),
                        transport_config=TransportConfig(enabled=True, water_enabled=False, initial_temperature_k=300.))
    rates = np.diag([1.5, -.75, .2]).astype(np.float32)
    x = to_np(sim.current_state.particle_positions)
    assign(sim.current_state.particle_velocities, (x - np.array([.5, .6, .5], np.float32)) @ rates.T)
    assign(sim.current_state.affine_velocities, np.tile(rates, (len(x), 1, 1)))
    return sim


@pytest.mark.parametrize("engine", ENGINES)
def test_invalid_pore_step_does_not_replace_the_last_valid_state(engine):
    api = Api(engine)
    sim = thermal_simulator(api, viscosity=1e4)
    x = to_np(sim.current_state.particle_positions)
    rates = -3000.0 * np.eye(3, dtype=np.float32)
    assign(sim.current_state.particle_velocities, (x - np.array([0.5, 0.6, 0.5], np.float32)) @ rates.T)
    assign(sim.current_state.affine_velocities, np.tile(rates, (len(x), 1, 1)))
    initial = sim.current_state
    with pytest.raises(RuntimeError, match="porosity left"):
        sim.Step()
    assert sim.current_state is initial
    assert sim.step_count == 0


@pytest.mark.parametrize("engine", ENGINES)
def test_gelatinization_from_particle_temperature_persists_on_cooling(engine):
    api = Api(engine)
    material = api.ding_material(MaterialConfig(), DingConfig(temperature_enabled=True))
    state = api.point(material)
    for T, yield_value, gelled in ((303.15, 1200., 0), (313.15, 400., 0), (353.15, 4000., 1), (293.15, 4000., 1)):
        assign(state.material_state.temperatures, [T])
        state = api.point_step(material, state, np.eye(3))
        np.testing.assert_allclose(ms(state, "yield_stresses"), yield_value, rtol=2e-6)
        assert ms(state, "gelled")[0] == gelled
