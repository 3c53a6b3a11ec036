"""Ideal-gas pore pressure and gas stress (the reference's ``physics/materials/gas.py:7-45``)."""

from __future__ import annotations

from ... import _lib, arrays

gas_constant = 8.31446261815324


def gas_pressure(moles, temperature, volume_ratio, porosity):
    """p = N R T / (J n) (host-side helper with the kernel's float64 formula)."""
    return moles * gas_constant * temperature / (volume_ratio * porosity)


def CombineGasStress(solid_stresses, gradients, porosities, moles, temperatures, total_stresses, error_flags,
                     ambient_pressure, initial_porosity, density, elastic_modulus, time_step, grid_spacing,
                     cfl_limit):
    n = gradients.shape[0]
    pitch = arrays.common_pitch(solid_stresses, gradients, total_stresses)
    _lib.call("bk_combine_gas_stress", n, pitch, arrays.ptr(solid_stresses), arrays.ptr(gradients),
              arrays.ptr(porosities), arrays.ptr(moles), arrays.ptr(temperatures), arrays.ptr(total_stresses),
              error_flags.data_ptr(), ambient_pressure, initial_porosity, arrays.ptr(density), elastic_modulus,
              time_step, grid_spacing, cfl_limit, _lib.stream_handle())


def RefreshGas(old_moles, new_moles, gradients, porosities, pressures, temperatures):
    n = gradients.shape[0]
    pitch = arrays.common_pitch(gradients)
    _lib.call("bk_refresh_gas", n, pitch, arrays.ptr(old_moles), arrays.ptr(new_moles), arrays.ptr(gradients),
              arrays.ptr(porosities), arrays.ptr(pressures), arrays.ptr(temperatures), _lib.stream_handle())
