"""Heat and water transport on the MPM grid (the reference's ``physics/thermal_water.py:41-367``).

One explicit split per substep: rebuild surface vertices -> boundary face areas
-> scalar P2G (volume, capacity, energy, water, boundary heat/loss/exchange) ->
7-point finite-volume diffusion with Robin boundary terms -> scalar G2P -> local
gas source -> water stress. Kernels run on the device behind the C ABI; this
module keeps the reference's ``TransportState`` fields and
``ThermalWaterTransport`` methods.
"""

from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np
import torch

from .. import _lib, arrays
from ..geometry import BoundaryFaces

GRID_FIELDS = ("volumes", "capacities", "energy", "water", "heat", "loss", "exchange", "temperatures",
               "saturations", "temperature_changes", "water_changes")


@dataclass
class TransportState:
    temperatures: torch.Tensor
    water_masses: torch.Tensor
    saturations: torch.Tensor
    water_losses: torch.Tensor
    heat_exchanges: torch.Tensor
    particle_masses: torch.Tensor


def AllocateTransportState(count, device):
    f64 = lambda: arrays.scalars(count, torch.float64, device)  # noqa: E731
    return TransportState(f64(), f64(), f64(), f64(), f64(), arrays.scalars(count, torch.float32, device))


def _origin(origin):
    return (_lib.F32 * 3)(*origin)


def scalar_params(config, simulation, settling):
    p = _lib.BkScalarParams()
    p.oven_temperature = config.oven_temperature_k
    p.tray_temperature = config.tray_temperature_k
    p.tray_transfer = 0.0 if settling else config.tray_heat_transfer
    p.surface_loss = 0.0 if settling else config.surface_water_loss
    p.water_density = config.water_density
    p.latent_heat = config.latent_heat
    p.water_enabled = int(config.water_enabled)
    p.origin[:] = list(simulation.grid_origin)
    p.spacing = simulation.grid_spacing
    p.resolution = simulation.grid_resolution
    return p


# ------------------------------------------------------------ kernel wrappers
def SurfaceAreas(vertices, faces, owners, exposed_areas, contact_areas, floor_height, contact_distance):
    _lib.call("bk_surface_areas", faces.shape[0], arrays.layout_pitch(vertices), arrays.ptr(vertices),
              faces.data_ptr(), owners.data_ptr(), exposed_areas.data_ptr(), contact_areas.data_ptr(),
              floor_height, contact_distance, _lib.stream_handle())


def ScalarToGrid(positions, gradients, reference_volumes, capacities, temperatures, water_masses, exposed, contact,
                 heat_parameter, params, grid, particle_heat, particle_loss, error_flags):
    fields = (_lib.P * 7)(*[grid[name].data_ptr() for name in GRID_FIELDS[:7]])
    n = positions.shape[0]
    _lib.call("bk_scalar_to_grid", n, arrays.common_pitch(positions, gradients), arrays.ptr(positions),
              arrays.ptr(gradients), arrays.ptr(reference_volumes), arrays.ptr(capacities), arrays.ptr(temperatures),
              arrays.ptr(water_masses), arrays.ptr(exposed), arrays.ptr(contact), arrays.ptr(heat_parameter),
              _lib.ctypes_ref(params), fields, arrays.ptr(particle_heat), arrays.ptr(particle_loss),
              error_flags.data_ptr(), _lib.stream_handle())


def GridFields(volumes, capacities, energy, water, temperatures, saturations, water_density):
    _lib.call("bk_grid_fields", volumes.shape[0], volumes.data_ptr(), capacities.data_ptr(), energy.data_ptr(),
              water.data_ptr(), temperatures.data_ptr(), saturations.data_ptr(), water_density,
              _lib.stream_handle())


def DiffuseGrid(volumes, capacities, temperatures, saturations, water, boundary_heat, boundary_loss,
                boundary_exchange, temperature_changes, water_changes, errors, conductivity, diffusivity,
                water_density, water_enabled, spacing, resolution, time_step):
    _lib.call("bk_diffuse_grid", volumes.shape[0], volumes.data_ptr(), capacities.data_ptr(),
              temperatures.data_ptr(), saturations.data_ptr(), water.data_ptr(), boundary_heat.data_ptr(),
              boundary_loss.data_ptr(), boundary_exchange.data_ptr(), temperature_changes.data_ptr(),
              water_changes.data_ptr(), errors.data_ptr(), conductivity, diffusivity, water_density,
              int(water_enabled), spacing, resolution, time_step, _lib.stream_handle())


def ScalarToParticles(positions, old_temperatures, old_water, old_losses, old_exchanges, dry_masses,
                      reference_volumes, gradients, node_water, temperature_changes, water_changes, particle_heat,
                      particle_loss, new_temperatures, material_temperatures, new_water, new_losses, new_exchanges,
                      new_masses, densities, saturations, water_density, origin, spacing, resolution, time_step,
                      error_flags):
    n = positions.shape[0]
    _lib.call("bk_scalar_to_particles", n, arrays.common_pitch(positions, gradients), arrays.ptr(positions),
              arrays.ptr(old_temperatures), arrays.ptr(old_water), arrays.ptr(old_losses), arrays.ptr(old_exchanges),
              arrays.ptr(dry_masses), arrays.ptr(reference_volumes), arrays.ptr(gradients), node_water.data_ptr(),
              temperature_changes.data_ptr(), water_changes.data_ptr(), arrays.ptr(particle_heat),
              arrays.ptr(particle_loss), arrays.ptr(new_temperatures), arrays.ptr(material_temperatures),
              arrays.ptr(new_water), arrays.ptr(new_losses), arrays.ptr(new_exchanges), arrays.ptr(new_masses),
              arrays.ptr(densities), arrays.ptr(saturations), water_density, _origin(origin), spacing, resolution,
              time_step, error_flags.data_ptr(), _lib.stream_handle())


def LocalGas(old_moles, old_temperatures, new_temperatures, new_moles, pressures, gradients, porosities, parameter,
             density, peak, width, time_step, produce):
    n = old_moles.shape[0]
    per_particle = int(parameter.shape[0] == n and n > 1)
    _lib.call("bk_local_gas", n, arrays.common_pitch(gradients), arrays.ptr(old_moles), arrays.ptr(old_temperatures),
              arrays.ptr(new_temperatures), arrays.ptr(new_moles), arrays.ptr(pressures), arrays.ptr(gradients),
              arrays.ptr(porosities), arrays.ptr(parameter), per_particle, density, peak, width, time_step,
              int(produce), _lib.stream_handle())


def WaterStress(gradients, saturations, old_stress, new_stress, initial_saturation, stiffness):
    n = gradients.shape[0]
    _lib.call("bk_water_stress", n, arrays.common_pitch(gradients, old_stress, new_stress), arrays.ptr(gradients),
              arrays.ptr(saturations), arrays.ptr(old_stress), arrays.ptr(new_stress), initial_saturation, stiffness,
              _lib.stream_handle())


def Saturations(water, reference_volumes, gradients, saturations, density):
    n = water.shape[0]
    _lib.call("bk_saturations", n, arrays.common_pitch(gradients), arrays.ptr(water), arrays.ptr(reference_volumes),
              arrays.ptr(gradients), arrays.ptr(saturations), density, _lib.stream_handle())


class ThermalWaterTransport:
    """Transport plugin: ``InitializeState``, ``Advance``, ``AddWaterStress``, ``FinishStep``."""

    def __init__(self, simulator, config):
        self.simulator = simulator
        self.config = config
        self.device = simulator.device
        samples = simulator.particle_samples
        density = simulator.material.material_config.density
        volumes = np.asarray(samples.reference_volumes, dtype=np.float64)
        self.reference_volumes = arrays.from_numpy(volumes.astype(np.float32), "f4", self.device)
        self.dry_masses = arrays.from_numpy((density - config.water_density * config.initial_saturation) * volumes,
                                            "f8", self.device)
        self.capacities = arrays.from_numpy(density * config.specific_heat * volumes, "f8", self.device)
        self.heat_transfer_parameter = torch.tensor([config.heat_transfer], dtype=torch.float32, device=self.device)
        self._zero_parameter = torch.zeros(1, dtype=torch.float32, device=self.device)
        faces, owners = BoundaryFaces(simulator.tet_mesh, samples)
        self.faces = torch.as_tensor(faces, device=self.device)
        self.owners = torch.as_tensor(owners, device=self.device)
        self.error_flags = torch.zeros(2, dtype=torch.int32, device=self.device)
        self.workspace = None
        self._grid = None

    def InitializeState(self, state):
        count = state.particle_positions.shape[0]
        c = self.config
        s = AllocateTransportState(count, self.device)
        s.temperatures.fill_(c.initial_temperature_k)
        volumes = np.asarray(self.simulator.particle_samples.reference_volumes, dtype=np.float64)
        arrays.assign(s.water_masses, c.water_density * c.initial_saturation * volumes)
        s.saturations.fill_(c.initial_saturation)
        arrays.assign(s.particle_masses, np.asarray(self.simulator.particle_samples.particle_masses, np.float32))
        state.transport_state = s
        self.error_flags.zero_()

    def grid_workspace(self):
        node_count = self.simulator.simulation_config.grid_resolution ** 3
        if self._grid is None or self._grid["volumes"].shape[0] != node_count:
            self._grid = {name: torch.zeros(node_count, dtype=torch.float64, device=self.device)
                          for name in GRID_FIELDS}
        return self._grid

    def Advance(self, state, time_step, settling=False, output=None, prepared_material=None, check=True):
        """Scalar transport for one substep; returns the prepared state (new T, water, gas).

        ``output``/``prepared_material`` let the simulator supply preallocated arrays;
        when omitted, fresh arrays are allocated like the reference does.
        """
        c = self.config
        sim = self.simulator.simulation_config
        count = state.particle_positions.shape[0]
        dev = self.device

        class Workspace:
            pass

        work = Workspace()
        work.heat_parameter = self._zero_parameter if settling else self.heat_transfer_parameter
        work.vertices = self.simulator.surface_vertices_buffer()
        self.simulator.mesh_binding.Reconstruct(state, work.vertices)
        ws = self.simulator.transport_particle_workspace()
        work.exposed, work.contact = ws["exposed"], ws["contact"]
        work.exposed.zero_()
        work.contact.zero_()
        floor = sim.grid_origin[1] + (sim.boundary_cells - 1) * sim.grid_spacing
        SurfaceAreas(work.vertices, self.faces, self.owners, work.exposed, work.contact, floor, c.contact_distance)
        grid = self.grid_workspace()
        for t in grid.values():
            t.zero_()
        work.grid = grid
        work.particle_heat, work.particle_loss = ws["particle_heat"], ws["particle_loss"]
        old = state.transport_state
        out = output if output is not None else AllocateTransportState(count, dev)
        if prepared_material is None:
            prepared_material = dict(temperatures=arrays.scalars(count, torch.float32, dev),
                                     reference_densities=arrays.scalars(count, torch.float32, dev),
                                     saturations=arrays.scalars(count, torch.float64, dev),
                                     gas_moles=arrays.scalars(count, torch.float64, dev),
                                     gas_pressures=arrays.scalars(count, torch.float64, dev))
        params = scalar_params(c, sim, settling)
        ScalarToGrid(state.particle_positions, state.deformation_gradients, self.reference_volumes, self.capacities,
                     old.temperatures, old.water_masses, work.exposed, work.contact, work.heat_parameter, params,
                     grid, work.particle_heat, work.particle_loss, self.simulator.error_flags)
        GridFields(grid["volumes"], grid["capacities"], grid["energy"], grid["water"], grid["temperatures"],
                   grid["saturations"], c.water_density)
        DiffuseGrid(grid["volumes"], grid["capacities"], grid["temperatures"], grid["saturations"], grid["water"],
                    grid["heat"], grid["loss"], grid["exchange"], grid["temperature_changes"], grid["water_changes"],
                    self.error_flags, 0.0 if settling else c.conductivity, 0.0 if settling else c.water_diffusivity,
                    c.water_density, c.water_enabled, sim.grid_spacing, sim.grid_resolution, time_step)
        if check:
            self.CheckState()
        prep_sat = prepared_material["saturations"]
        ScalarToParticles(state.particle_positions, old.temperatures, old.water_masses, old.water_losses,
                          old.heat_exchanges, self.dry_masses, self.reference_volumes, state.deformation_gradients,
                          grid["water"], grid["temperature_changes"], grid["water_changes"], work.particle_heat,
                          work.particle_loss, out.temperatures, prepared_material["temperatures"], out.water_masses,
                          out.water_losses, out.heat_exchanges, out.particle_masses,
                          prepared_material["reference_densities"], prep_sat, c.water_density, sim.grid_origin,
                          sim.grid_spacing, sim.grid_resolution, time_step, self.simulator.error_flags)
        material = self.simulator.material
        material_state = replace(state.material_state, temperatures=prepared_material["temperatures"],
                                 reference_densities=prepared_material["reference_densities"])
        if material.ding_config.gas_enabled:
            material_state.gas_moles = prepared_material["gas_moles"]
            material_state.gas_pressures = prepared_material["gas_pressures"]
            d = material.ding_config
            LocalGas(state.material_state.gas_moles, old.temperatures, out.temperatures, material_state.gas_moles,
                     material_state.gas_pressures, state.deformation_gradients, state.material_state.porosities,
                     material.production_parameter, material.material_config.density, d.gas_reaction_temperature_k,
                     d.gas_reaction_width_k, time_step, int(not settling))
        prepared_transport = replace(out, saturations=prep_sat)
        work.prepared = replace(state, material_state=material_state, transport_state=prepared_transport)
        work.output = out
        self.workspace = work
        return work.prepared

    def FlagMessage(self, flags):
        if flags[0] or flags[1]:
            return ("Heat/water explicit stability bound exceeded; reduce time_step; no temperature or water "
                    "clipping is applied")
        return None

    def CheckState(self):
        message = self.FlagMessage(self.error_flags.tolist())
        if message:
            raise RuntimeError(message)

    def AddWaterStress(self, state, stress, output=None):
        out = output if output is not None else arrays.like(stress)
        c = self.config
        WaterStress(state.deformation_gradients, state.transport_state.saturations, stress, out, c.initial_saturation,
                    c.water_stress if c.water_enabled else 0.0)
        if self.workspace is not None:
            self.workspace.stress_before_water = stress
        return out

    def FinishStep(self, prepared, output):
        out = self.workspace.output if self.workspace is not None else prepared.transport_state
        output.transport_state = out
        Saturations(out.water_masses, self.reference_volumes, output.deformation_gradients, out.saturations,
                    self.config.water_density)
