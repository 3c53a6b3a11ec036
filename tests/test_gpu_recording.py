"""The recorder's device measurement against the oracle (oracle/measure.py, a restatement of
experiments/recording.py:46-112), the Step() hook and the run folder, and the reference's
invalid-pore-step test (tests/test_ding_thermal.py:193-209)."""
from dataclasses import replace

import numpy as np
import pytest

from baking_b200.config import ExperimentConfig, RunConfig

pytestmark = pytest.mark.gpu


def _host(t):
    from baking_b200 import arrays
    return arrays.to_numpy(t)


def oracle_measure(sim):
    from baking_b200.physics.materials.ding import DingMaterial
    from oracle.measure import core_mask, measure
    sim.UpdateMesh()
    st = sim.current_state
    ding = gas = transport = None
    if isinstance(sim.material, DingMaterial):
        ms = st.material_state
        ding = {k: _host(getattr(ms, k)) for k in ("temperatures", "porosities", "gelled", "yield_stresses",
                                                   "viscosities")}
        if sim.material.ding_config.gas_enabled:
            gas = {k: _host(getattr(ms, k)) for k in ("gas_moles", "gas_pressures")}
    if sim.transport is not None:
        t = st.transport_state
        c = sim.transport.config
        V0 = np.asarray(sim.particle_samples.reference_volumes, np.float64)
        transport = {k: _host(getattr(t, k)) for k in ("temperatures", "water_masses", "saturations",
                                                       "water_losses", "heat_exchanges")}
        transport.update(capacities=_host(sim.transport.capacities), owners=_host(sim.transport.owners),
                         core=core_mask(sim.particle_samples.particle_positions, sim.tet_mesh.vertex_positions),
                         initial_temperature=c.initial_temperature_k,
                         initial_water=c.water_density * c.initial_saturation * V0.sum())
    return measure(_host(sim.vertex_positions), sim.tet_mesh.tet_indices, _host(st.deformation_gradients),
                   np.asarray(sim.particle_samples.reference_volumes, np.float64), ding, gas, transport)


def compare(device, oracle):
    for key, value in oracle.items():
        got = device[key]
        if isinstance(value, int):
            assert got == value, key
        elif key == "energy_balance_error_j":
            # energy - initial energy - heat exchanged: a cancellation of float64 sums, compared at
            # the rounding level of the thermal energy (sums in another order)
            assert got == pytest.approx(value, abs=1e-11 * abs(oracle["thermal_energy_j"])), key
        else:
            # float32 reference volumes and float64 sums in another order; material temperatures
            # averaged in float64
            assert got == pytest.approx(value, rel=2e-6, abs=1e-9 * max(1.0, abs(value))), key


def test_measure_matches_oracle_gas_transport(tmp_path):
    from baking_b200.recording import SimulationRecorder
    from tests.scenes import baking_cube, set_velocity_field
    sim, rates = baking_cube("cuda")
    set_velocity_field(sim, rates)
    sim.Advance(6)
    config = replace(ExperimentConfig(), run=replace(RunConfig(), log_path=str(tmp_path)))
    rec = SimulationRecorder(sim, config)
    m = rec.Measure()
    compare(m, oracle_measure(sim))
    assert m["step"] == 6 and m["phase"] == "baking" and m["inverted_tets"] == 0


def test_measure_elastic_model(tmp_path):
    from baking_b200.recording import SimulationRecorder
    from tests.test_gpu_adjoint import neo_hookean_sim
    sim = neo_hookean_sim()
    sim.Advance(3)
    config = replace(ExperimentConfig(), run=replace(RunConfig(), log_path=str(tmp_path)))
    m = SimulationRecorder(sim, config).Measure()
    assert "porosity_mean" not in m and "water_mass_kg" not in m
    compare(m, oracle_measure(sim))


def test_step_records_and_finish_writes_the_run(tmp_path):
    import json
    from baking_b200.recording import SimulationRecorder
    from tests.scenes import build_transport
    sim = build_transport("cuda", gas=True)
    config = replace(ExperimentConfig(), run=replace(RunConfig(), log_path=str(tmp_path), snapshot_interval=2))
    rec = SimulationRecorder(sim, config)
    sim.result_recorder = rec
    for _ in range(4):
        sim.Step()
    assert len(rec.expansion_history) == 5 and [h["step"] for h in rec.expansion_history] == [0, 1, 2, 3, 4]
    assert [s for s, _ in rec.pending_snapshots] == [0, 2, 4]
    compare(rec.last_measurement, oracle_measure(sim))
    path = rec.Finish()
    summary = json.loads((path / "summary.json").read_text())
    assert summary["status"] == "completed" and summary["final"]["step"] == 4
    for name in ("expansion_history.csv", "height_history.csv", "material_history.csv",
                 "thermal_water_history.csv", "final_state.npz", "final_surface.obj", "snapshot_0000004.npz"):
        assert (path / name).exists(), name
    assert rec.Finish() == path


def test_invalid_pore_step_does_not_replace_or_record_the_last_valid_state(tmp_path):
    """A strongly compressed porous cube: the step's porosity leaves [0, 1); Step() raises before
    committing, and nothing is recorded or written."""
    from baking_b200.recording import SimulationRecorder
    from tests.test_gpu_adjoint_transport import thermal_sim
    from tests.scenes import assign, to_np
    sim = thermal_sim(1e4, short_curve=False)
    x = to_np(sim.current_state.particle_positions)
    rates = -3000.0 * np.eye(3, dtype=np.float32)
    assign(sim.current_state.particle_velocities, (x - np.array([0.5, 0.6, 0.5], np.float32)) @ rates.T)
    assign(sim.current_state.affine_velocities, np.tile(rates, (len(x), 1, 1)))
    config = replace(ExperimentConfig(), run=replace(RunConfig(), log_path=str(tmp_path / "results")))
    rec = SimulationRecorder(sim, config)
    sim.result_recorder = rec
    initial = sim.current_state
    with pytest.raises(RuntimeError, match="porosity left"):
        sim.Step()
    assert sim.current_state is initial
    assert sim.step_count == 0 and len(rec.expansion_history) == 1
    assert not (tmp_path / "results").exists()
