"""CPU restatement of the recorder's per-step measurement -- test infrastructure.

The checker for ``bk_measure_state`` / ``baking_b200.recording.SimulationRecorder.Measure``: the
statistics of SimulationRecorder.Measure (experiments/recording.py:46-112) computed with numpy in
float64 from host copies of the same arrays, in the reference's formulas (reference-volume
weighted particle volume, gas and pore volume; capacity-weighted mean temperature; surface-owner
and initial-core temperature means; water and energy balances; axis-aligned mesh extents; summed
absolute tet volumes and inverted tets).
"""
from __future__ import annotations

import numpy as np


def signed_volumes(vertices, tets):
    """geometry/mesh_validation.py ComputeSignedVolumes: det of the three edge rows / 6."""
    corners = np.asarray(vertices, np.float64)[np.asarray(tets)]
    return np.linalg.det(corners[:, 1:] - corners[:, :1]) / 6.0


def core_mask(sample_positions, mesh_vertices):
    """Particles whose sampled position lies within 0.4 of the largest distance from the
    reference mesh centroid (recording.py:80-86)."""
    center = np.mean(mesh_vertices, axis=0)
    radius = np.linalg.norm(np.asarray(sample_positions) - center, axis=1)
    core = radius < 0.4 * radius.max()
    return core if core.any() else radius == radius.min()


def measure(vertices, tets, F, V0, ding=None, gas=None, transport=None):
    """``ding``: dict(temperatures, porosities, gelled, yield_stresses, viscosities);
    ``gas``: dict(gas_moles, gas_pressures); ``transport``: dict(temperatures, water_masses,
    saturations, water_losses, heat_exchanges, capacities, owners, core, initial_temperature,
    initial_water). Returns the measurement values (without the step/time keys)."""
    vertices = np.asarray(vertices, np.float64)
    F = np.asarray(F, np.float64)
    V0 = np.asarray(V0, np.float64)
    if not np.isfinite(vertices).all() or not np.isfinite(F).all():
        raise ValueError("Cannot record nonfinite simulation state")
    vols = signed_volumes(vertices, tets)
    J = np.linalg.det(F)
    extent = np.ptp(vertices, axis=0)
    out = {}
    if ding is not None:
        por = np.asarray(ding["porosities"], np.float64)
        out.update(temperature_k=float(np.asarray(ding["temperatures"], np.float64).mean()),
                   porosity_min=float(por.min()), porosity_mean=float(por.mean()), porosity_max=float(por.max()),
                   yield_stress_pa=float(ding["yield_stresses"][0]), viscosity_pa3_s=float(ding["viscosities"][0]),
                   gelled_fraction=float(np.asarray(ding["gelled"]).mean()))
        if gas is not None:
            N = np.asarray(gas["gas_moles"], np.float64)
            p = np.asarray(gas["gas_pressures"], np.float64)
            out.update(gas_total_mol=float(np.dot(V0, N)), gas_pressure_min_pa=float(p.min()),
                       gas_pressure_max_pa=float(p.max()), gas_pressure_mean_pa=float(p.mean()),
                       pore_volume_m3=float(np.dot(V0, J * por)))
    if transport is not None:
        T = np.asarray(transport["temperatures"], np.float64)
        W = np.asarray(transport["water_masses"], np.float64)
        s = np.asarray(transport["saturations"], np.float64)
        c = np.asarray(transport["capacities"], np.float64)
        surface = np.zeros(len(W), dtype=bool)
        surface[np.asarray(transport["owners"])] = True
        core = np.asarray(transport["core"])
        energy = float(np.dot(c, T))
        exchange = float(np.asarray(transport["heat_exchanges"], np.float64).sum())
        losses = float(np.asarray(transport["water_losses"], np.float64).sum())
        out.update(temperature_min_k=float(T.min()), temperature_max_k=float(T.max()),
                   temperature_mean_k=float(np.average(T, weights=c)),
                   temperature_surface_k=float(T[surface].mean()), temperature_core_k=float(T[core].mean()),
                   water_mass_kg=float(W.sum()), water_lost_kg=losses,
                   water_balance_error_kg=float(W.sum() + losses - transport["initial_water"]),
                   saturation_min=float(s.min()), saturation_max=float(s.max()), saturation_mean=float(s.mean()),
                   thermal_energy_j=energy, heat_exchange_j=exchange,
                   energy_balance_error_j=float(energy - transport["initial_temperature"] * c.sum() - exchange))
    out.update(length_x_m=float(extent[0]), width_z_m=float(extent[2]), height_y_m=float(extent[1]),
               particle_volume_m3=float(np.dot(V0, J)), mesh_volume_m3=float(np.abs(vols).sum()),
               inverted_tets=int(np.count_nonzero(vols <= 0)), invalid_particles=int(np.count_nonzero(J <= 0)))
    return out
