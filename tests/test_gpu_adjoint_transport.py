"""Hand-written adjoint of the transport substep (Ding with thermal-water transport, gas off)
against finite differences and the reference's heated porous MPM known answer
(tests/test_ding_thermal.py:160-190 with BuildThermalSimulator of :213-225).

The directional checks use the helpers of test_gpu_adjoint.py: <dL/dtheta, delta> against central
differences of the forward run, one output array at a time.
"""
from dataclasses import replace

import numpy as np
import pytest

from baking_b200.config import DingConfig, MaterialConfig, SimulationConfig, TransportConfig
from baking_b200.geometry import CreateDemoMesh, SampleParticles
from tests.test_gpu_adjoint import STRAIN_RATES, _coherent, _delta, directional_check

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


# ----------------------------------------------------------------- known answer
def thermal_sim(viscosity, short_curve=True):
    """BuildThermalSimulator: demo cube, Ding with temperature and porosity 0.2, transport with water
    off from 300 K, strain-rate field; short_curve: yield 5 Pa and dt 1 ms, else 100 Pa and 0.1 ms."""
    from baking_b200.physics.mpm import MpmSimulator
    from tests.scenes import assign, to_np
    mesh = CreateDemoMesh(1)
    sim = MpmSimulator(mesh, SampleParticles(mesh, 1000.0, 4),
                       replace(SimulationConfig(), device_name="cuda:0", time_step=0.001 if short_curve else 0.0001,
                               gravity=(0.0, 0.0, 0.0)),
                       MaterialConfig(model="ding2019"),
                       ding_config=DingConfig(temperature_enabled=True, porosity=0.2,
                                              yield_stress=5.0 if short_curve else 100.0, viscosity=viscosity),
                       transport_config=TransportConfig(enabled=True, water_enabled=False,
                                                        initial_temperature_k=300.0))
    st = sim.current_state
    x = to_np(st.particle_positions)
    assign(st.particle_velocities, ((x - np.array([0.5, 0.6, 0.5], np.float32)) @ STRAIN_RATES.T).astype(np.float32))
    assign(st.affine_velocities, np.tile(STRAIN_RATES, (len(x), 1, 1)))
    return sim


def thermal_viscosity_loss(value, grad):
    """5 substeps, loss = mean tau_00 of the final state."""
    torch = _torch()
    from baking_b200.physics.adjoint import Rollout
    sim = thermal_sim(value)
    eta = torch.tensor([value], dtype=torch.float32, device="cuda", requires_grad=grad)
    out = Rollout(sim, 5, checkpoint_every=2, viscosity_parameter=eta)
    loss = out["kirchhoff_stresses"][:, 0, 0].mean()
    sim.CheckState()
    if grad:
        loss.backward()
        return float(loss.detach()), float(eta.grad[0])
    return float(loss.detach()), None


def test_heated_porous_mpm_viscosity_gradient_known_answer():
    _, gradient = thermal_viscosity_loss(1000.0, True)
    fd = (thermal_viscosity_loss(1010.0, False)[0] - thermal_viscosity_loss(990.0, False)[0]) / 20.0
    assert abs(fd) > 1e-7
    np.testing.assert_allclose(gradient, fd, rtol=0.03, atol=1e-7)


# ------------------------------------------------------------ directional checks
def heated_sim(water=True):
    """A prestrained porous Ding cube in a hot oven: strong surface heating, conduction, water
    diffusion, surface water loss with latent heat, water stress, temperature-dependent viscosity."""
    from baking_b200.physics.mpm import MpmSimulator
    from tests.scenes import assign, to_np
    mesh = CreateDemoMesh(2)
    transport = TransportConfig(enabled=True, water_enabled=water, initial_temperature_k=300.0,
                                oven_temperature_k=480.0, heat_transfer=2000.0, conductivity=20.0,
                                specific_heat=100.0, water_diffusivity=1e-8, surface_water_loss=1e-5,
                                latent_heat=2.0e4 if water else 0.0)
    sim = MpmSimulator(mesh, SampleParticles(mesh, 1000.0, 4),
                       replace(SimulationConfig(), device_name="cuda:0", time_step=0.001, gravity=(0.0, 0.0, 0.0)),
                       MaterialConfig(model="ding2019"),
                       ding_config=DingConfig(yield_stress=50.0, viscosity=1000.0, porosity=0.3,
                                              temperature_enabled=True),
                       transport_config=transport)
    rng = np.random.default_rng(5)
    n = sim.particle_data.particle_count
    st = sim.current_state
    x = to_np(st.particle_positions)
    assign(st.particle_velocities, ((x - np.array([0.5, 0.6, 0.5], np.float32)) @ STRAIN_RATES.T).astype(np.float32))
    assign(st.affine_velocities, np.tile(STRAIN_RATES, (n, 1, 1)))
    Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    Q *= np.sign(np.linalg.det(Q))
    Fe = (Q @ np.diag([1.01, 0.995, 1.003]) @ Q.T)[None] + 0.003 * rng.standard_normal((n, 3, 3))
    assign(st.material_state.elastic_gradients, Fe.astype(np.float32))
    assign(st.deformation_gradients, Fe.astype(np.float32))
    tau = 20.0 * rng.standard_normal((n, 3, 3))
    assign(st.material_state.kirchhoff_stresses, (tau + tau.transpose(0, 2, 1)).astype(np.float32))
    t = st.transport_state
    assign(t.temperatures, 300.0 + 5.0 * rng.random(n))
    if water:
        assign(t.water_masses, to_np(t.water_masses) * (1.0 + 0.1 * rng.random(n)))
    return sim


def _shape(sim, name):
    n = sim.particle_data.particle_count
    return {"velocities": (n, 3), "positions": (n, 3), "deformation_gradients": (n, 3, 3),
            "transport_temperatures": (n,), "water_masses": (n,), "heat_transfer_parameter": (1,),
            "viscosity_parameter": (1,)}[name]


@pytest.mark.parametrize("name,scale,eps", [
    ("transport_temperatures", 2.0, 0.5), ("heat_transfer_parameter", 200.0, 0.5), ("velocities", 0.02, 0.5),
    ("positions", 0.002, 0.5), ("deformation_gradients", 0.002, 0.5), ("viscosity_parameter", 100.0, 0.5)])
def test_heated_directional(name, scale, eps):
    sim = heated_sim()
    directional_check(heated_sim, 5, name, _delta(_shape(sim, name), 23, scale), eps)


def test_water_mass_directional():
    sim = heated_sim()
    w0 = sim.current_state.transport_state.water_masses.clone()
    delta = 0.05 * w0 * _coherent(tuple(w0.shape), 29)
    directional_check(heated_sim, 5, "water_masses", delta, 0.5)


def test_dry_heating_directional():
    """Water off: heat transfer and conduction alone drive the material temperature."""
    make = lambda: heated_sim(water=False)  # noqa: E731
    sim = make()
    directional_check(make, 5, "transport_temperatures", _delta(_shape(sim, "transport_temperatures"), 31, 2.0), 0.5)


def test_checkpoint_interval_does_not_change_transport_gradients():
    """Every checkpoint interval reuses the per-substep grids differently; the node fields and the
    node scratch must be back at zero after each reverse step for the gradients to agree."""
    torch = _torch()
    from baking_b200.physics.adjoint import Rollout
    grads = []
    for every in (1, 3, 16):
        sim = heated_sim()
        T = sim.current_state.transport_state.temperatures.clone().requires_grad_(True)
        v = sim.current_state.particle_velocities.clone().requires_grad_(True)
        out = Rollout(sim, 7, checkpoint_every=every, transport_temperatures=T, velocities=v)
        (out["kirchhoff_stresses"][:, 0, 1].sum() + out["transport_temperatures"].sum() +
         1e3 * out["water_masses"].sum()).backward()
        grads.append((T.grad.clone(), v.grad.clone()))
    for k in range(2):
        scale = float(grads[0][k].abs().max())
        for other in grads[1:]:
            torch.testing.assert_close(grads[0][k], other[k], rtol=1e-3, atol=1e-4 * scale)


def test_backward_leaves_the_simulator_state():
    """The reverse sweep re-runs substeps on its own grids and surface buffers: the simulator then
    continues exactly as one whose Rollout was not differentiated."""
    torch = _torch()
    from baking_b200.physics.adjoint import Rollout
    finals = []
    for differentiate in (False, True):
        sim = heated_sim()
        T = sim.current_state.transport_state.temperatures.clone().requires_grad_(differentiate)
        out = Rollout(sim, 4, checkpoint_every=2, transport_temperatures=T)
        if differentiate:
            out["transport_temperatures"].sum().backward()
        sim.AdvanceUnchecked(3)
        st = sim.current_state
        finals.append([st.particle_positions.clone(), st.transport_state.temperatures.clone(),
                       st.transport_state.water_masses.clone(), st.transport_state.heat_exchanges.clone()])
    for a, b in zip(*finals):  # float atomics may sum in another order between the two runs
        torch.testing.assert_close(a, b, rtol=1e-5, atol=1e-6 * float(a.abs().max()))


# ------------------------------------------------------------------- gas mode
def gassy_sim(per_particle=True):
    """The heated cube in gas mode: coupled end-state porosity, gas source around its reaction
    temperature (per-particle rates), gas-pressure stress, water transport."""
    from baking_b200.physics.mpm import MpmSimulator
    from tests.scenes import assign, to_np
    mesh = CreateDemoMesh(2)
    transport = TransportConfig(enabled=True, initial_temperature_k=325.0, oven_temperature_k=480.0,
                                heat_transfer=2000.0, conductivity=20.0, specific_heat=100.0,
                                water_diffusivity=1e-8, surface_water_loss=1e-5)
    ding = DingConfig(yield_stress=50.0, viscosity=1000.0, porosity=0.3, temperature_enabled=True, gas_enabled=True,
                      gas_initial_pressure_pa=1000.0, gas_ambient_pressure_pa=1000.0, gas_production_rate=0.005)
    sim = MpmSimulator(mesh, SampleParticles(mesh, 1000.0, 4),
                       replace(SimulationConfig(), device_name="cuda:0", time_step=0.001, gravity=(0.0, 0.0, 0.0)),
                       MaterialConfig(model="ding2019"), ding_config=ding, transport_config=transport)
    rng = np.random.default_rng(7)
    n = sim.particle_data.particle_count
    st = sim.current_state
    x = to_np(st.particle_positions)
    assign(st.particle_velocities, ((x - np.array([0.5, 0.6, 0.5], np.float32)) @ STRAIN_RATES.T).astype(np.float32))
    assign(st.affine_velocities, np.tile(STRAIN_RATES, (n, 1, 1)))
    Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    Q *= np.sign(np.linalg.det(Q))
    Fe = (Q @ np.diag([1.01, 0.995, 1.003]) @ Q.T)[None] + 0.003 * rng.standard_normal((n, 3, 3))
    assign(st.material_state.elastic_gradients, Fe.astype(np.float32))
    assign(st.deformation_gradients, Fe.astype(np.float32))
    tau = 20.0 * rng.standard_normal((n, 3, 3))
    assign(st.material_state.kirchhoff_stresses, (tau + tau.transpose(0, 2, 1)).astype(np.float32))
    assign(st.transport_state.temperatures, 320.0 + 10.0 * rng.random(n))
    if per_particle:
        sim.SetGasSourceRates((0.003 + 0.004 * rng.random(n)).astype(np.float32))
    return sim


def _gas_shape(sim, name):
    n = sim.particle_data.particle_count
    return {"velocities": (n, 3), "deformation_gradients": (n, 3, 3), "elastic_gradients": (n, 3, 3),
            "porosities": (n,), "transport_temperatures": (n,), "viscosity_parameter": (1,),
            "young_modulus": (1,), "gas_source_rates": (n,)}[name]


@pytest.mark.parametrize("name,scale,eps", [
    ("gas_source_rates", 0.002, 0.5), ("transport_temperatures", 2.0, 0.5), ("porosities", 0.01, 0.5),
    ("elastic_gradients", 0.002, 0.5), ("deformation_gradients", 0.002, 0.5), ("velocities", 0.02, 0.5),
    ("viscosity_parameter", 100.0, 0.5), ("young_modulus", 1000.0, 1.0)])
def test_gas_directional(name, scale, eps):
    sim = gassy_sim()
    directional_check(gassy_sim, 5, name, _delta(_gas_shape(sim, name), 37, scale), eps)


def test_gas_moles_directional():
    sim = gassy_sim()
    N0 = sim.current_state.material_state.gas_moles.clone()
    directional_check(gassy_sim, 5, "gas_moles", 0.2 * N0 * _coherent(tuple(N0.shape), 41), 0.5)


def test_shared_gas_rate_directional():
    """One production parameter for every particle (the reference's scalar)."""
    make = lambda: gassy_sim(per_particle=False)  # noqa: E731
    directional_check(make, 5, "gas_source_rates", _delta((1,), 43, 0.002), 0.5)


def test_private_surface_buffers_use_the_vertex_pitch():
    """The reverse sweep's own vertex buffer is written by the vertex kernel in plane layout with
    the surface's vertex pitch; a row-major buffer would be written past its end."""
    from baking_b200 import arrays
    from baking_b200.physics.adjoint import Rollout
    sim = heated_sim()
    T = sim.current_state.transport_state.temperatures.clone().requires_grad_(True)
    Rollout(sim, 2, transport_temperatures=T)["transport_temperatures"].sum().backward()
    verts = sim._buffers["rollout"]["transport"]["surface_vertices"]
    assert arrays.layout_pitch(verts) == sim._engine.surface.vertex_pitch
    assert verts.shape == sim.surface_vertices_buffer().shape
