"""The recorder measurement oracle (oracle/measure.py) on cases with known answers, and the C-ABI
struct the device reduction takes."""
import ctypes

import numpy as np
import pytest

from oracle.measure import core_mask, measure, signed_volumes

UNIT_TET = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float64)


def test_signed_volume_orientation():
    assert signed_volumes(UNIT_TET, [[0, 1, 2, 3]])[0] == pytest.approx(1 / 6)
    assert signed_volumes(UNIT_TET, [[0, 2, 1, 3]])[0] == pytest.approx(-1 / 6)


def test_known_measurements():
    F = np.stack([np.diag([2.0, 1.0, 1.0]), np.diag([1.0, 1.0, -0.5])])
    V0 = np.array([0.1, 0.3])
    verts = UNIT_TET * np.array([2.0, 3.0, 4.0])
    ding = dict(temperatures=[300.0, 310.0], porosities=[0.2, 0.4], gelled=[0, 1], yield_stresses=[5.0, 6.0],
                viscosities=[7.0, 8.0])
    gas = dict(gas_moles=[1.0, 2.0], gas_pressures=[100.0, 300.0])
    transport = dict(temperatures=[300.0, 400.0], water_masses=[1.0, 3.0], saturations=[0.2, 0.6],
                     water_losses=[0.5, 0.0], heat_exchanges=[10.0, 20.0], capacities=[1.0, 3.0], owners=[1],
                     core=np.array([True, False]), initial_temperature=300.0, initial_water=5.0)
    m = measure(verts, [[0, 1, 2, 3], [0, 2, 1, 3]], F, V0, ding, gas, transport)
    assert m["particle_volume_m3"] == pytest.approx(0.1 * 2.0 - 0.3 * 0.5)
    assert m["invalid_particles"] == 1
    assert m["mesh_volume_m3"] == pytest.approx(2 * 24 / 6) and m["inverted_tets"] == 1
    assert (m["length_x_m"], m["height_y_m"], m["width_z_m"]) == (2.0, 3.0, 4.0)
    assert m["temperature_k"] == 305.0 and m["porosity_mean"] == pytest.approx(0.3)
    assert m["gelled_fraction"] == 0.5 and m["yield_stress_pa"] == 5.0 and m["viscosity_pa3_s"] == 7.0
    assert m["gas_total_mol"] == pytest.approx(0.7) and m["gas_pressure_mean_pa"] == 200.0
    assert m["pore_volume_m3"] == pytest.approx(0.1 * 2.0 * 0.2 - 0.3 * 0.5 * 0.4)
    assert m["temperature_mean_k"] == pytest.approx(375.0)
    assert m["temperature_surface_k"] == 400.0 and m["temperature_core_k"] == 300.0
    assert m["water_balance_error_kg"] == pytest.approx(4.0 + 0.5 - 5.0)
    assert m["energy_balance_error_j"] == pytest.approx(1500.0 - 1200.0 - 30.0)


def test_nonfinite_state_is_rejected():
    with pytest.raises(ValueError, match="nonfinite"):
        measure(UNIT_TET, [[0, 1, 2, 3]], np.full((1, 3, 3), np.nan), [1.0])


def test_core_mask_falls_back_to_the_innermost_particles():
    pts = np.array([[0.0, 0, 0], [1.0, 0, 0]])  # both 0.5 from the centroid: none within 0.4 of it
    assert core_mask(pts, pts).tolist() == [True, True]
    pts = np.array([[0.5, 0, 0], [0.0, 0, 0], [1.0, 0, 0]])
    assert core_mask(pts, pts).tolist() == [True, False, False]


def test_measure_inputs_struct_matches_the_header():
    from baking_b200.recording import SLOTS, BkMeasureInputs
    assert ctypes.sizeof(BkMeasureInputs) == 21 * 8
    assert len(SLOTS) == 35
