"""Ding 2019 viscoplastic dough skeleton (the reference's ``physics/materials/ding.py:33-327``).

The return map (trial Fe* = (I + dt C) Fe, float64 SVD, Hencky stress, scalar
overstress Newton solve, projection, isochoric/porosity volume correction,
Fp = Fe^-1 F, porosity = det Fp - 1 + n0 or the coupled end-state porosity in gas
mode) runs in the sm_100a kernel behind ``bk_update_ding``; this module keeps the
reference's ``DingState`` fields and ``DingMaterial`` plugin methods.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from ... import _lib, arrays
from .elastic import ElasticMaterial
from .gas import CombineGasStress, RefreshGas, gas_constant


@dataclass
class DingState:
    """Gas content is mol per initial m^3; pressures are absolute Pa."""
    elastic_gradients: torch.Tensor
    plastic_gradients: torch.Tensor
    kirchhoff_stresses: torch.Tensor
    return_residuals: torch.Tensor
    porosities: torch.Tensor
    temperatures: torch.Tensor
    gelled: torch.Tensor
    yield_stresses: torch.Tensor
    viscosities: torch.Tensor
    gas_moles: torch.Tensor
    gas_pressures: torch.Tensor
    porosity_residuals: torch.Tensor
    reference_densities: torch.Tensor


def TemperatureFactor(temperature_value, temperature_knots, factor_values):
    """Piecewise-linear factor table with constant extrapolation (host side, float64)."""
    return float(np.interp(temperature_value, temperature_knots, factor_values))


def PorosityCoefficient(porosity):
    """a(n) = 9 / (4 log(1/n)^2 (3.5 n + 1)); 0 at n = 0 (von Mises limit)."""
    return 0.0 if porosity <= 0 else 9.0 / (4.0 * math.log(1.0 / porosity) ** 2 * (3.5 * porosity + 1.0))


def ding_params(material_config, ding_config, time_step):
    p = _lib.BkDingParams()
    p.coupled_porosity = int(ding_config.gas_enabled)
    p.temperature_enabled = int(ding_config.temperature_enabled)
    p.shear_modulus = material_config.shear_modulus
    p.lame_lambda = material_config.lame_lambda
    p.yield_stress = ding_config.yield_stress
    p.initial_porosity = ding_config.porosity
    p.time_step = time_step
    p.temperature_knots[:] = list(ding_config.temperature_knots_k)
    p.yield_factors[:] = list(ding_config.yield_factors)
    p.viscosity_factors[:] = list(ding_config.viscosity_factors)
    return p


def UpdateDing(old_state, total_gradients, affine_velocities, new_state, viscosity_parameter, error_flags, params,
               local_temperatures):
    n = total_gradients.shape[0]
    pitch = arrays.common_pitch(old_state.elastic_gradients, total_gradients, affine_velocities,
                                new_state.elastic_gradients, new_state.plastic_gradients,
                                new_state.kirchhoff_stresses)
    _lib.call("bk_update_ding", n, pitch, arrays.ptr(old_state.elastic_gradients), arrays.ptr(old_state.porosities),
              arrays.ptr(old_state.gelled), arrays.ptr(total_gradients), arrays.ptr(affine_velocities),
              arrays.ptr(new_state.elastic_gradients), arrays.ptr(new_state.plastic_gradients),
              arrays.ptr(new_state.kirchhoff_stresses), arrays.ptr(new_state.return_residuals),
              arrays.ptr(new_state.porosities), arrays.ptr(new_state.temperatures), arrays.ptr(new_state.gelled),
              arrays.ptr(new_state.yield_stresses), arrays.ptr(new_state.viscosities),
              arrays.ptr(viscosity_parameter), error_flags.data_ptr(), arrays.ptr(new_state.porosity_residuals),
              _lib.ctypes_ref(params), arrays.ptr(local_temperatures), _lib.stream_handle())


def AllocateDingState(count, device, pitch=None):
    f32 = lambda: arrays.scalars(count, torch.float32, device)  # noqa: E731
    f64 = lambda: arrays.scalars(count, torch.float64, device)  # noqa: E731
    return DingState(
        elastic_gradients=arrays.mat33s(count, device=device, pitch=pitch),
        plastic_gradients=arrays.mat33s(count, device=device, pitch=pitch),
        kirchhoff_stresses=arrays.mat33s(count, device=device, pitch=pitch),
        return_residuals=f32(), porosities=f32(), temperatures=f32(),
        gelled=arrays.scalars(count, torch.int32, device), yield_stresses=f32(), viscosities=f32(),
        gas_moles=f64(), gas_pressures=f64(), porosity_residuals=f32(), reference_densities=f32())


class DingMaterial(ElasticMaterial):
    def __init__(self, material_config, ding_config, device_name="cuda", requires_grad=False,
                 initial_temperature_k=293.15):
        super().__init__(material_config)
        ding_config.Validate()
        self.device = _lib.require_cuda(device_name)
        self.initial_temperature_k = initial_temperature_k
        self.ding_config = ding_config
        self.requires_grad = requires_grad
        self.viscosity_parameter = torch.tensor([ding_config.viscosity], dtype=torch.float32, device=self.device)
        self.production_parameter = torch.tensor([ding_config.gas_production_rate], dtype=torch.float32,
                                                 device=self.device)
        self.error_flags = torch.zeros(3, dtype=torch.int32, device=self.device)
        self.pressure_coefficient = PorosityCoefficient(ding_config.porosity)
        self.Reset()

    def Reset(self):
        self.error_flags.zero_()

    def InitialValues(self):
        c = self.ding_config
        T = self.initial_temperature_k
        gelled = int(c.temperature_enabled and T >= c.temperature_knots_k[3])
        yf = TemperatureFactor(T, c.temperature_knots_k, c.yield_factors) if c.temperature_enabled else 1.0
        vf = TemperatureFactor(T, c.temperature_knots_k, c.viscosity_factors) if c.temperature_enabled else 1.0
        moles = c.gas_initial_pressure_pa * c.porosity / (gas_constant * T) if c.gas_enabled else 0.0
        return dict(temperature=T, gelled=gelled, yield_stress=c.yield_stress * yf,
                    viscosity=float(self.viscosity_parameter[0].item()) * vf, moles=moles,
                    pressure=c.gas_initial_pressure_pa if c.gas_enabled else 0.0)

    def InitializeState(self, particle_state, values=None):
        count = particle_state.particle_positions.shape[0]
        device = particle_state.particle_positions.device
        pitch = arrays.layout_pitch(particle_state.deformation_gradients)
        values = values or self.InitialValues()
        s = AllocateDingState(count, device, pitch)
        eye = torch.eye(3, device=device)
        s.elastic_gradients.copy_(eye)
        s.plastic_gradients.copy_(eye)
        s.porosities.fill_(self.ding_config.porosity)
        s.temperatures.fill_(values["temperature"])
        s.gelled.fill_(values["gelled"])
        s.yield_stresses.fill_(values["yield_stress"])
        s.viscosities.fill_(values["viscosity"])
        s.gas_moles.fill_(values["moles"])
        s.gas_pressures.fill_(values["pressure"])
        s.reference_densities.fill_(self.material_config.density)
        particle_state.material_state = s

    def ComputeStress(self, particle_state, kirchhoff_stresses, error_flags):
        state = particle_state.material_state
        if not self.ding_config.gas_enabled:
            kirchhoff_stresses.copy_(state.kirchhoff_stresses)
            return
        self.LaunchGasStress(particle_state, kirchhoff_stresses)
        self.CheckState()

    def LaunchGasStress(self, particle_state, kirchhoff_stresses):
        state = particle_state.material_state
        sim = getattr(self, "simulation_config", None)
        mc = self.material_config
        CombineGasStress(state.kirchhoff_stresses, particle_state.deformation_gradients, state.porosities,
                         state.gas_moles, state.temperatures, kirchhoff_stresses, self.error_flags,
                         self.ding_config.gas_ambient_pressure_pa, self.ding_config.porosity,
                         state.reference_densities, mc.lame_lambda + 2 * mc.shear_modulus,
                         sim.time_step if sim else 0.0, sim.grid_spacing if sim else 1.0,
                         sim.cfl_limit if sim else 0.4)

    def GasWaveSpeed(self, particle_state):
        s = particle_state.material_state
        n = s.porosities.double()
        bulk = s.gas_pressures * (1 + (1 - self.ding_config.porosity + n) / n)
        J = torch.linalg.det(particle_state.deformation_gradients.double())
        K = self.material_config.lame_lambda + 2 * self.material_config.shear_modulus
        return float(torch.sqrt((K + bulk) * J / s.reference_densities.double()).max().item())

    def FlagMessage(self, flags):
        if flags[2]:
            return "Gas acoustic CFL exceeds the explicit limit; reduce time_step. Pressure is not capped"
        if flags[1]:
            return ("Coupled porosity return has no resolved interior solution; reduce dt/loading. "
                    "No pore-volume clipping or closed-pore law is applied")
        if flags[0]:
            return ("Ding porosity left [0, 1); no constitutive clamping is applied. Reduce dt or loading; "
                    "the paper gives no closure beyond this domain")
        return None

    def CheckState(self):
        message = self.FlagMessage(self.error_flags.tolist())
        if message:
            raise RuntimeError(message)

    def AdvanceState(self, input_state, output_state, time_step):
        if output_state.material_state is None:
            self.InitializeState(output_state)
        old, new = input_state.material_state, output_state.material_state
        params = ding_params(self.material_config, self.ding_config, time_step)
        UpdateDing(old, output_state.deformation_gradients, output_state.affine_velocities, new,
                   self.viscosity_parameter, self.error_flags, params, old.temperatures)
        new.reference_densities.copy_(old.reference_densities)
        if self.ding_config.gas_enabled:
            RefreshGas(old.gas_moles, new.gas_moles, output_state.deformation_gradients, new.porosities,
                       new.gas_pressures, new.temperatures)
