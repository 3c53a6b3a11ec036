"""CPU oracle of ``MpmSimulator.Step`` -- test infrastructure only.

Drives the C restatement (``ora.py``) of every reference kernel in the order of
``physics/mpm.py:163-225`` with the host logic of ``physics/materials/ding.py:224-327``,
``physics/materials/elastic.py:29-49``, ``physics/thermal_water.py:263-367`` and
``physics/mpm.py:24-308``. State lives in numpy arrays in the reference's
layouts; every step allocates fresh output arrays like the reference's history mode.
Only the tests, the smoke check and the CPU-baseline leg of bench.py use this.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np

from baking_b200.config import DingConfig
from baking_b200.geometry import BoundaryFaces, ComputeSignedVolumes, MeshBindingTables_build

from . import ora

GAS_CONSTANT = 8.31446261815324


@dataclass
class ParticleState:
    particle_positions: np.ndarray
    particle_velocities: np.ndarray
    deformation_gradients: np.ndarray
    affine_velocities: np.ndarray
    material_state: object = None
    transport_state: object = None


@dataclass
class ParticleData:
    particle_masses: np.ndarray
    reference_volumes: np.ndarray
    particle_count: int


@dataclass
class DingState:
    elastic_gradients: np.ndarray
    plastic_gradients: np.ndarray
    kirchhoff_stresses: np.ndarray
    return_residuals: np.ndarray
    porosities: np.ndarray
    temperatures: np.ndarray
    gelled: np.ndarray
    yield_stresses: np.ndarray
    viscosities: np.ndarray
    gas_moles: np.ndarray
    gas_pressures: np.ndarray
    porosity_residuals: np.ndarray
    reference_densities: np.ndarray


@dataclass
class TransportState:
    temperatures: np.ndarray
    water_masses: np.ndarray
    saturations: np.ndarray
    water_losses: np.ndarray
    heat_exchanges: np.ndarray
    particle_masses: np.ndarray


def AllocateState(n):
    return ParticleState(ora.f32(n, 3), ora.f32(n, 3), ora.f32(n, 3, 3), ora.f32(n, 3, 3))


def CreateParticleState(samples, initial_velocity=(0.0, 0.0, 0.0)):
    n = len(samples.particle_positions)
    v0 = np.asarray(initial_velocity, dtype=np.float32)
    if v0.shape != (3,) or not np.isfinite(v0).all():
        raise ValueError("initial_velocity must have three finite components")
    state = AllocateState(n)
    state.particle_positions[:] = samples.particle_positions.astype(np.float32)
    state.particle_velocities[:] = v0
    state.deformation_gradients[:] = np.eye(3, dtype=np.float32)
    data = ParticleData(np.ascontiguousarray(samples.particle_masses, dtype=np.float32),
                        np.ascontiguousarray(samples.reference_volumes, dtype=np.float32), n)
    return state, data


def TemperatureFactor(value, knots, factors):
    return float(np.interp(value, knots, factors))


class ElasticMaterial:
    def __init__(self, material_config):
        material_config.Validate()
        self.material_config = material_config

    def ComputeStress(self, particle_state, kirchhoff_stresses, error_flags):
        ora.compute_elastic_stress(particle_state.deformation_gradients, kirchhoff_stresses,
                                   self.material_config.shear_modulus, self.material_config.lame_lambda,
                                   error_flags)

    def AdvanceState(self, input_state, output_state, time_step):
        output_state.material_state = None


class DingMaterial(ElasticMaterial):
    def __init__(self, material_config, ding_config, requires_grad=False, initial_temperature_k=293.15):
        super().__init__(material_config)
        ding_config.Validate()
        self.initial_temperature_k = initial_temperature_k
        self.ding_config = ding_config
        self.viscosity_parameter = np.array([ding_config.viscosity], dtype=np.float32)
        self.production_parameter = np.array([ding_config.gas_production_rate], dtype=np.float32)
        self.error_flags = ora.i32(3)
        n0 = ding_config.porosity
        self.pressure_coefficient = 0.0 if n0 == 0 else 9.0 / (4.0 * math.log(1.0 / n0) ** 2 * (3.5 * n0 + 1.0))

    def Reset(self):
        self.error_flags[:] = 0

    def InitializeState(self, particle_state):
        n = len(particle_state.particle_positions)
        cfg = self.ding_config
        T = self.initial_temperature_k
        gelled = int(cfg.temperature_enabled and T >= cfg.temperature_knots_k[3])
        yf = TemperatureFactor(T, cfg.temperature_knots_k, cfg.yield_factors) if cfg.temperature_enabled else 1.0
        vf = TemperatureFactor(T, cfg.temperature_knots_k, cfg.viscosity_factors) if cfg.temperature_enabled else 1.0
        eye = np.tile(np.eye(3, dtype=np.float32), (n, 1, 1))
        moles = cfg.gas_initial_pressure_pa * cfg.porosity / (GAS_CONSTANT * T) if cfg.gas_enabled else 0.0
        particle_state.material_state = DingState(
            elastic_gradients=eye.copy(), plastic_gradients=eye.copy(), kirchhoff_stresses=ora.f32(n, 3, 3),
            return_residuals=ora.f32(n), porosities=np.full(n, cfg.porosity, np.float32),
            temperatures=np.full(n, T, np.float32), gelled=np.full(n, gelled, np.int32),
            yield_stresses=np.full(n, cfg.yield_stress * yf, np.float32),
            viscosities=np.full(n, float(self.viscosity_parameter[0]) * vf, np.float32),
            gas_moles=np.full(n, moles, np.float64),
            gas_pressures=np.full(n, cfg.gas_initial_pressure_pa if cfg.gas_enabled else 0.0, np.float64),
            porosity_residuals=ora.f32(n),
            reference_densities=np.full(n, self.material_config.density, np.float32))

    def ComputeStress(self, particle_state, kirchhoff_stresses, error_flags):
        state = particle_state.material_state
        if not self.ding_config.gas_enabled:
            kirchhoff_stresses[:] = state.kirchhoff_stresses
            return
        sim = getattr(self, "simulation_config", None)
        mc = self.material_config
        ora.combine_gas_stress(state.kirchhoff_stresses, particle_state.deformation_gradients, state.porosities,
                               state.gas_moles, state.temperatures, kirchhoff_stresses, self.error_flags,
                               self.ding_config.gas_ambient_pressure_pa, self.ding_config.porosity,
                               state.reference_densities, mc.lame_lambda + 2 * mc.shear_modulus,
                               sim.time_step if sim else 0.0, sim.grid_spacing if sim else 1.0,
                               sim.cfl_limit if sim else 0.4)
        self.CheckState()

    def GasWaveSpeed(self, particle_state):
        s = particle_state.material_state
        n = s.porosities.astype(np.float64)
        bulk = s.gas_pressures * (1 + (1 - self.ding_config.porosity + n) / n)
        J = np.linalg.det(particle_state.deformation_gradients.astype(np.float64))
        K = self.material_config.lame_lambda + 2 * self.material_config.shear_modulus
        return float(np.sqrt((K + bulk) * J / s.reference_densities).max())

    def CheckState(self):
        flags = self.error_flags
        if flags[2]:
            raise RuntimeError("Gas acoustic CFL exceeds the explicit limit; reduce time_step. Pressure is not capped")
        if flags[1]:
            raise RuntimeError("Coupled porosity return has no resolved interior solution; reduce dt/loading. "
                               "No pore-volume clipping or closed-pore law is applied")
        if flags[0]:
            raise RuntimeError("Ding porosity left [0, 1); no constitutive clamping is applied. Reduce dt or "
                               "loading; the paper gives no closure beyond this domain")

    def AdvanceState(self, input_state, output_state, time_step):
        n = len(output_state.particle_positions)
        if output_state.material_state is None:
            self.InitializeState(output_state)
        old, new = input_state.material_state, output_state.material_state
        cfg, mc = self.ding_config, self.material_config
        params = ora.ding_params(cfg.gas_enabled, cfg.temperature_enabled, mc.shear_modulus, mc.lame_lambda,
                                 cfg.yield_stress, cfg.porosity, time_step, cfg.temperature_knots_k,
                                 cfg.yield_factors, cfg.viscosity_factors)
        ora.update_ding(old.elastic_gradients, old.porosities, old.gelled, output_state.deformation_gradients,
                        output_state.affine_velocities, new.elastic_gradients, new.plastic_gradients,
                        new.kirchhoff_stresses, new.return_residuals, new.porosities, new.temperatures,
                        new.gelled, new.yield_stresses, new.viscosities, self.viscosity_parameter,
                        self.error_flags, new.porosity_residuals, params, old.temperatures)
        new.reference_densities[:] = old.reference_densities
        if cfg.gas_enabled:
            ora.refresh_gas(old.gas_moles, new.gas_moles, output_state.deformation_gradients, new.porosities,
                            new.gas_pressures, new.temperatures)
        del n


class ThermalWaterTransport:
    def __init__(self, simulator, config):
        self.simulator = simulator
        self.config = config
        samples = simulator.particle_samples
        density = simulator.material.material_config.density
        self.reference_volumes = np.ascontiguousarray(samples.reference_volumes, dtype=np.float32)
        self.dry_masses = np.ascontiguousarray(
            (density - config.water_density * config.initial_saturation) * samples.reference_volumes, np.float64)
        self.capacities = np.ascontiguousarray(density * config.specific_heat * samples.reference_volumes,
                                               np.float64)
        self.heat_transfer_parameter = np.array([config.heat_transfer], dtype=np.float32)
        faces, owners = BoundaryFaces(simulator.tet_mesh, samples)
        self.faces = np.ascontiguousarray(faces, np.int32)
        self.owners = np.ascontiguousarray(owners, np.int32)
        self.error_flags = ora.i32(2)
        self.workspace = None

    def InitializeState(self, state):
        n = len(state.particle_positions)
        c = self.config
        V0 = self.simulator.particle_samples.reference_volumes
        state.transport_state = TransportState(
            np.full(n, c.initial_temperature_k, np.float64),
            np.ascontiguousarray(c.water_density * c.initial_saturation * V0, np.float64),
            np.full(n, c.initial_saturation, np.float64), ora.f64(n), ora.f64(n),
            np.ascontiguousarray(self.simulator.particle_samples.particle_masses, np.float32))
        self.error_flags[:] = 0

    def Advance(self, state, time_step, settling=False):
        c = self.config
        sim = self.simulator.simulation_config
        n = len(state.particle_positions)
        R = sim.grid_resolution
        nn = R ** 3

        class Workspace:
            pass

        w = Workspace()
        w.heat_parameter = ora.f32(1) if settling else self.heat_transfer_parameter
        w.vertices = ora.f32(len(self.simulator.tet_mesh.vertex_positions), 3)
        self.simulator.mesh_binding_reconstruct(state, w.vertices)
        w.exposed, w.contact = ora.f64(n), ora.f64(n)
        floor = sim.grid_origin[1] + (sim.boundary_cells - 1) * sim.grid_spacing
        ora.surface_areas(w.vertices, self.faces, self.owners, w.exposed, w.contact, floor, c.contact_distance)
        g = {name: ora.f64(nn) for name in ("volumes", "capacities", "energy", "water", "heat", "loss", "exchange",
                                            "temperatures", "saturations", "temperature_changes",
                                            "water_changes")}
        w.grid = g
        w.particle_heat, w.particle_loss = ora.f64(n), ora.f64(n)
        old = state.transport_state
        out = TransportState(ora.f64(n), ora.f64(n), ora.f64(n), ora.f64(n), ora.f64(n), ora.f32(n))
        mat_T, densities = ora.f32(n), ora.f32(n)
        params = ora.scalar_params(c.oven_temperature_k, c.tray_temperature_k,
                                   0.0 if settling else c.tray_heat_transfer,
                                   0.0 if settling else c.surface_water_loss, c.water_density, c.latent_heat,
                                   c.water_enabled, sim.grid_origin, sim.grid_spacing, R)
        ora.scalar_to_grid(state.particle_positions, state.deformation_gradients, self.reference_volumes,
                           self.capacities, old.temperatures, old.water_masses, w.exposed, w.contact,
                           w.heat_parameter, params, g, w.particle_heat, w.particle_loss,
                           self.simulator.error_flags)
        ora.grid_fields(g["volumes"], g["capacities"], g["energy"], g["water"], g["temperatures"],
                        g["saturations"], c.water_density)
        ora.diffuse_grid(g["volumes"], g["capacities"], g["temperatures"], g["saturations"], g["water"], g["heat"],
                         g["loss"], g["exchange"], g["temperature_changes"], g["water_changes"], self.error_flags,
                         0.0 if settling else c.conductivity, 0.0 if settling else c.water_diffusivity,
                         c.water_density, c.water_enabled, sim.grid_spacing, R, time_step)
        if self.error_flags[0] or self.error_flags[1]:
            raise RuntimeError("Heat/water explicit stability bound exceeded; reduce time_step; no temperature or "
                               "water clipping is applied")
        ora.scalar_to_particles(state.particle_positions, old.temperatures, old.water_masses, old.water_losses,
                                old.heat_exchanges, self.dry_masses, self.reference_volumes,
                                state.deformation_gradients, g["water"], g["temperature_changes"],
                                g["water_changes"], w.particle_heat, w.particle_loss, out.temperatures, mat_T,
                                out.water_masses, out.water_losses, out.heat_exchanges, out.particle_masses,
                                densities, out.saturations, c.water_density, sim.grid_origin, sim.grid_spacing, R,
                                time_step, self.simulator.error_flags)
        material_state = replace(state.material_state, temperatures=mat_T, reference_densities=densities)
        material = self.simulator.material
        if material.ding_config.gas_enabled:
            material_state.gas_moles, material_state.gas_pressures = ora.f64(n), ora.f64(n)
            dc = material.ding_config
            ora.local_gas(state.material_state.gas_moles, old.temperatures, out.temperatures,
                          material_state.gas_moles, material_state.gas_pressures, state.deformation_gradients,
                          state.material_state.porosities, material.production_parameter,
                          material.material_config.density, dc.gas_reaction_temperature_k,
                          dc.gas_reaction_width_k, time_step, int(not settling))
        w.prepared = replace(state, material_state=material_state, transport_state=out)
        self.workspace = w
        return w.prepared

    def AddWaterStress(self, state, stress):
        out = ora.f32(len(state.particle_positions), 3, 3)
        c = self.config
        ora.water_stress(state.deformation_gradients, state.transport_state.saturations, stress, out,
                         c.initial_saturation, c.water_stress if c.water_enabled else 0.0)
        return out

    def FinishStep(self, prepared, output):
        n = len(output.particle_positions)
        output.transport_state = replace(prepared.transport_state, saturations=ora.f64(n))
        ora.saturations(output.transport_state.water_masses, self.reference_volumes,
                        output.deformation_gradients, output.transport_state.saturations, self.config.water_density)


class OracleSimulator:
    """The reference substep on the CPU oracle, with the reference's constructor and methods."""

    def __init__(self, tet_mesh, particle_samples, simulation_config, material_config,
                 initial_velocity=(0.0, 0.0, 0.0), retain_history=False, ding_config=None, transport_config=None,
                 gas_source_rates=None):
        simulation_config.Validate(material_config)
        self.tet_mesh = tet_mesh
        self.particle_samples = particle_samples
        self.simulation_config = simulation_config
        self.material = ElasticMaterial(material_config)
        if material_config.model == "ding2019":
            self.material = DingMaterial(material_config, ding_config or DingConfig(), retain_history)
            self.material.simulation_config = simulation_config
            if gas_source_rates is not None:
                self.material.production_parameter = np.ascontiguousarray(gas_source_rates, np.float32)
        if (isinstance(self.material, DingMaterial) and self.material.ding_config.gas_enabled
                and not (transport_config and transport_config.enabled)):
            raise ValueError("Ding gas simulation requires transport.enabled=true; prescribed temperature "
                             "schedules were removed")
        self.initial_velocity = initial_velocity
        self.retain_history = retain_history
        self.ValidateInitialDomain()
        self.binding = MeshBindingTables_build(tet_mesh, particle_samples)
        self._binding_arrays = (np.ascontiguousarray(tet_mesh.vertex_positions, np.float32),
                                self.binding.binding_offsets, self.binding.binding_particles,
                                np.ascontiguousarray(self.binding.binding_weights, np.float32),
                                np.ascontiguousarray(self.binding.reference_offsets, np.float32))
        self.transport = None
        if transport_config is not None and transport_config.enabled:
            transport_config.Validate(material_config)
            self.material.initial_temperature_k = transport_config.initial_temperature_k
            self.error_flags = ora.i32(2)
            self.transport = ThermalWaterTransport(self, transport_config)
        self.Reset()

    # ------------------------------------------------------------ helpers
    def SetGasSourceRates(self, rates):
        self.material.production_parameter = np.ascontiguousarray(np.asarray(rates, np.float32).reshape(-1))

    def mesh_binding_reconstruct(self, state, out):
        ref, offsets, particles, weights, offs = self._binding_arrays
        ora.reconstruct_mesh_vertices(state.particle_positions, state.deformation_gradients, ref, offsets,
                                      particles, weights, offs, out)

    def Masses(self, state=None):
        state = self.current_state if state is None else state
        return state.transport_state.particle_masses if state.transport_state is not None else \
            self.particle_data.particle_masses

    def ValidateInitialDomain(self):
        s = self.simulation_config
        origin = np.asarray(s.grid_origin)
        lower = origin + (s.boundary_cells - 1) * s.grid_spacing
        upper = origin + (s.grid_resolution - s.boundary_cells) * s.grid_spacing
        points = np.concatenate([self.tet_mesh.vertex_positions, self.particle_samples.particle_positions])
        if np.any(points < lower) or np.any(points > upper):
            raise ValueError(f"model must initially fit inside {lower} .. {upper}")

    @property
    def settling_steps(self):
        if self.transport is None:
            return 0
        if self._baking_start_step is not None and self._baking_start_step > 0:
            return self._baking_start_step
        return int(math.ceil(self.transport.config.settling_duration_s / self.simulation_config.time_step - 1e-10))

    @property
    def IsSettling(self):
        return (self.transport is not None and self.transport.config.settling_duration_s > 0
                and self._baking_start_step is None)

    def Reset(self):
        if isinstance(self.material, DingMaterial):
            self.material.Reset()
        self.current_state, self.particle_data = CreateParticleState(self.particle_samples, self.initial_velocity)
        if isinstance(self.material, DingMaterial):
            self.material.InitializeState(self.current_state)
        if self.transport is not None:
            self.transport.InitializeState(self.current_state)
        R = self.simulation_config.grid_resolution
        self.node_count = R ** 3
        self.grid_masses, self.grid_momenta, self.grid_velocities = ora.f32(R ** 3), ora.f32(R ** 3, 3), \
            ora.f32(R ** 3, 3)
        self.kirchhoff_stresses = ora.f32(self.particle_data.particle_count, 3, 3)
        self.vertex_positions = np.ascontiguousarray(self.tet_mesh.vertex_positions, np.float32)
        self.error_flags = ora.i32(2)
        self.step_count = 0
        self._baking_start_step = None if (self.transport is not None
                                           and self.transport.config.settling_duration_s > 0) else 0
        self.mesh_step_count = 0

    def Step(self):
        sim = self.simulation_config
        was_settling = self.IsSettling
        original = self.current_state
        state = original
        if self.transport is not None:
            state = self.transport.Advance(state, sim.time_step, settling=was_settling)
        n = self.particle_data.particle_count
        output = AllocateState(n)
        R = sim.grid_resolution
        self.grid_masses[:] = 0
        self.grid_momenta[:] = 0
        self.grid_velocities[:] = 0
        stress = ora.f32(n, 3, 3)
        self.material.ComputeStress(state, stress, self.error_flags)
        if self.transport is not None:
            stress = self.transport.AddWaterStress(state, stress)
        ora.particle_to_grid(state.particle_positions, state.particle_velocities, state.affine_velocities, stress,
                             self.Masses(state), self.particle_data.reference_volumes, self.grid_masses,
                             self.grid_momenta, sim.grid_origin, sim.grid_spacing, R, sim.time_step,
                             self.error_flags)
        ora.update_grid(self.grid_masses, self.grid_momenta, self.grid_velocities, R, sim.boundary_cells,
                        sim.gravity, sim.time_step)
        ora.grid_to_particle(state.particle_positions, state.deformation_gradients, self.grid_velocities,
                             output.particle_positions, output.particle_velocities, output.affine_velocities,
                             output.deformation_gradients, sim.grid_origin, sim.grid_spacing, R, sim.time_step,
                             self.error_flags)
        self.material.AdvanceState(state, output, sim.time_step)
        if isinstance(self.material, DingMaterial):
            self.material.CheckState()
        if self.transport is not None:
            self.transport.FinishStep(state, output)
        self.current_state = output
        self.step_count += 1
        if was_settling:
            self._UpdateSettlingFixed()

    def _UpdateSettlingFixed(self):
        if self.transport.config.settling_auto:
            raise NotImplementedError("the oracle restates fixed-duration settling only")
        if self.step_count >= self.settling_steps:
            self._baking_start_step = self.step_count

    def Advance(self, step_count):
        if step_count < 1:
            raise ValueError("step_count must be positive")
        for _ in range(step_count):
            self.Step()
        return self.CheckState()

    def UpdateMesh(self, force_update=False):
        if force_update or self.mesh_step_count != self.step_count:
            out = ora.f32(len(self.tet_mesh.vertex_positions), 3)
            self.mesh_binding_reconstruct(self.current_state, out)
            self.vertex_positions = out
            self.mesh_step_count = self.step_count

    def CheckState(self):
        flags = self.error_flags
        if flags[0]:
            raise RuntimeError("nonpositive/nonfinite J; reduce dt or inspect loading and sampling")
        if flags[1]:
            raise RuntimeError("particle stencil left the grid; enlarge the domain or reduce dt")
        st = self.current_state
        x, v, F, Cm = st.particle_positions, st.particle_velocities, st.deformation_gradients, st.affine_velocities
        if not all(np.isfinite(a).all() for a in (x, v, F, Cm)):
            raise RuntimeError("nonfinite particle state; simulation stopped")
        J = np.linalg.det(F)
        if J.min() <= 0.0:
            raise RuntimeError("inverted particle deformation; reduce dt or loading")
        sim = self.simulation_config
        gpos = (x - np.array(sim.grid_origin)) / sim.grid_spacing
        if np.any(gpos < 0.5) or np.any(gpos >= sim.grid_resolution - 1.5):
            raise RuntimeError("particle outside valid grid stencil")
        masses = self.Masses().astype(np.float64)
        vmax = float(np.linalg.norm(v, axis=1).max())
        wave = self.material.material_config.wave_speed
        if isinstance(self.material, DingMaterial) and self.material.ding_config.gas_enabled:
            wave = max(wave, self.material.GasWaveSpeed(st))
        if self.transport is not None and self.transport.config.water_enabled:
            ww = self.transport.config.water_stress * st.transport_state.saturations * J / \
                st.material_state.reference_densities
            wave = float(np.sqrt(wave * wave + ww.max()))
        cfl = (vmax + wave) * sim.time_step / sim.grid_spacing
        if cfl > sim.cfl_limit:
            raise RuntimeError(f"estimated CFL={cfl:.3f} > {sim.cfl_limit}; reduce dt")
        if isinstance(self.material, DingMaterial):
            self.material.CheckState()
            ms = st.material_state
            if not np.isfinite(ms.elastic_gradients).all() or not np.isfinite(ms.plastic_gradients).all():
                raise RuntimeError("nonfinite Ding internal state")
            if float(ms.return_residuals.max()) > 1e-4:
                raise RuntimeError("Ding local return mapping did not converge")
        self.UpdateMesh()
        return {
            "step_count": self.step_count,
            "simulation_time": self.step_count * sim.time_step,
            "particle_count": self.particle_data.particle_count,
            "particle_volume_m3": float(np.dot(self.particle_samples.reference_volumes, J)),
            "total_mass": float(masses.sum()),
            "grid_mass": float(self.grid_masses.sum(dtype=np.float64)),
            "minimum_j": float(J.min()), "maximum_j": float(J.max()), "maximum_speed": vmax,
            "kinetic_energy": float(0.5 * np.sum(masses * np.sum(v.astype(np.float64) ** 2, axis=1))),
            "estimated_cfl": cfl,
            "unmapped_mesh_vertices": self.binding.unmapped_vertex_count,
            "inverted_mesh_tets": int(np.count_nonzero(
                ComputeSignedVolumes(self.vertex_positions.astype(np.float64), self.tet_mesh.tet_indices) <= 0)),
        }
