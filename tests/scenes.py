"""Scene builders shared by the oracle (CPU) and device (GPU) tests.

They restate the reference tests' set-ups (tests/test_transport.py:12-20
BuildTransport, tests/test_gas.py:333-341 BuildGasSimulator,
tests/test_ding_thermal.py:418-430 BuildThermalSimulator) for either engine.
"""
from dataclasses import replace

import numpy as np

from baking_b200.config import DingConfig, MaterialConfig, SimulationConfig, TransportConfig
from baking_b200.geometry import CreateDemoMesh, SampleParticles


def engine_class(engine):
    if engine == "oracle":
        from oracle.sim import OracleSimulator
        return OracleSimulator
    from baking_b200.physics.mpm import MpmSimulator
    return MpmSimulator


def build_transport(engine, config=None, history=False, spacing=0.025, dt=0.0001, subdivisions=2, gas=False):
    mesh = CreateDemoMesh(subdivisions)
    return engine_class(engine)(
        mesh, SampleParticles(mesh, 1000., 4),
        replace(SimulationConfig(), device_name="cpu" if engine == "oracle" else "cuda:0", time_step=dt,
                gravity=(0., 0., 0.), grid_spacing=spacing, grid_resolution=int(round(1 / spacing))),
        MaterialConfig(model="ding2019", young_modulus=10000.), retain_history=history,
        ding_config=DingConfig(gas_enabled=gas, porosity=0.2 if gas else 0., gas_production_rate=0.001,
                               temperature_enabled=True),
        transport_config=config or TransportConfig(enabled=True))


def build_gas(engine, rate=0.005, dt=0.0005, history=False):
    mesh = CreateDemoMesh(1)
    config = DingConfig(gas_enabled=True, porosity=0.2, yield_stress=20., viscosity=1e5,
                        gas_initial_pressure_pa=1000., gas_ambient_pressure_pa=1000., gas_production_rate=rate)
    return engine_class(engine)(
        mesh, SampleParticles(mesh, 1000., 4),
        replace(SimulationConfig(), device_name="cpu" if engine == "oracle" else "cuda:0", time_step=dt,
                gravity=(0., 0., 0.)),
        MaterialConfig(model="ding2019", young_modulus=10000.), retain_history=history, ding_config=config,
        transport_config=TransportConfig(enabled=True, water_enabled=False, initial_temperature_k=333.15,
                                         conductivity=0., heat_transfer=0., tray_heat_transfer=0.))


def baking_cube(engine, subdivisions=2, gravity=(0., -9.81, 0.), dt=1e-4, seed=0):
    """Demo cube with Ding + temperature + gas + water transport, gravity and a seeded strain-rate field."""
    mesh = CreateDemoMesh(subdivisions)
    sim = engine_class(engine)(
        mesh, SampleParticles(mesh, 1000., 4),
        replace(SimulationConfig(), device_name="cpu" if engine == "oracle" else "cuda:0", time_step=dt,
                gravity=gravity),
        MaterialConfig(model="ding2019", young_modulus=2e4),
        ding_config=DingConfig(gas_enabled=True, porosity=0.2, yield_stress=200., viscosity=1e6,
                               temperature_enabled=True, gas_production_rate=0.01),
        transport_config=TransportConfig(enabled=True, initial_temperature_k=330.0, oven_temperature_k=480.,
                                         heat_transfer=2000., conductivity=20., specific_heat=100.,
                                         water_diffusivity=1e-8, surface_water_loss=1e-5))
    rng = np.random.default_rng(seed)
    rates = np.diag([1.5, -0.75, 0.2]).astype(np.float32) + 0.1 * rng.standard_normal((3, 3)).astype(np.float32)
    return sim, rates


def set_velocity_field(sim, rates, center=(0.5, 0.6, 0.5)):
    """v = rates (x - center), C = rates (the reference tests' imposed deformation)."""
    st = sim.current_state
    x = to_np(st.particle_positions)
    v = ((x - np.asarray(center, np.float32)) @ rates.T).astype(np.float32)
    assign(st.particle_velocities, v)
    assign(st.affine_velocities, np.tile(rates, (len(x), 1, 1)))


def to_np(a):
    if isinstance(a, np.ndarray):
        return a
    return a.detach().cpu().numpy()


def assign(a, values):
    values = np.asarray(values)
    if isinstance(a, np.ndarray):
        a[...] = values.astype(a.dtype).reshape(a.shape)
    else:
        import torch
        a.copy_(torch.as_tensor(values).to(a.dtype).reshape(a.shape))
