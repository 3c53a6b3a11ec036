"""Batched independent simulators under one CUDA graph (BatchedSimulators) against the same bodies
advanced one by one through MpmSimulator.AdvanceUnchecked."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bodies(prestrain=(0.0, 0.0)):
    from baking_b200 import scenes
    return scenes.dough_batch(6, seed=3, particles=(5_000, 20_000), resolutions=(32, 48), prestrain=prestrain)


@pytest.mark.parametrize("prestrain", [(0.0, 0.0), (0.04, 0.1)])
def test_graph_replay_matches_individual_advance(prestrain):
    from baking_b200 import scenes
    from baking_b200.batch import BatchedSimulators
    scs = bodies(prestrain)
    batched = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    single = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    batch = BatchedSimulators(batched, streams=4).capture()   # capture runs two substeps
    batch.Advance(10)
    for sim in single:
        sim.AdvanceUnchecked(12)
    for b, s, sc in zip(batched, single, scs):
        assert b.step_count == s.step_count == 12
        xb = b.current_state.particle_positions.cpu().numpy()
        xs = s.current_state.particle_positions.cpu().numpy()
        dx = sc.simulation.grid_spacing
        np.testing.assert_allclose(xb, xs, rtol=0, atol=1e-4 * dx)
        Tb = b.current_state.transport_state.temperatures.cpu().numpy()
        Ts = s.current_state.transport_state.temperatures.cpu().numpy()
        np.testing.assert_allclose(Tb, Ts, rtol=1e-6)
        assert Tb.max() > sc.transport.initial_temperature_k   # the oven is heating each body
    for st in batch.CheckState():
        assert st["step_count"] == 12


def test_snapshot_restore_repeats_a_run():
    from baking_b200 import scenes
    from baking_b200.batch import BatchedSimulators, RestoreStates, SnapshotStates
    sims = [scenes.make_simulator(s, diagnostics="lean") for s in bodies((0.04, 0.1))]
    saved = SnapshotStates(sims)
    batch = BatchedSimulators(sims, streams=4).capture()
    batch.Advance(4)
    first = [s.current_state.particle_positions.cpu().numpy().copy() for s in sims]
    RestoreStates(sims, saved)
    batch.Advance(6)   # capture ran 2 substeps before the first replay; 2 + 4 == 6
    for s, x in zip(sims, first):
        np.testing.assert_allclose(s.current_state.particle_positions.cpu().numpy(), x, rtol=0, atol=1e-6)
