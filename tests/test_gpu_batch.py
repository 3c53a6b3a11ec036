"""Batched independent simulators under one CUDA graph (BatchedSimulators) against the same bodies
advanced one by one through MpmSimulator.AdvanceUnchecked."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bodies(prestrain=(0.0, 0.0)):
    from baking_b200 import scenes
    return scenes.dough_batch(6, seed=3, particles=(5_000, 20_000), resolutions=(32, 48), prestrain=prestrain)


def _compare(batched, single, scs, steps, porosity_atol=1e-6):
    for b, s, sc in zip(batched, single, scs):
        assert b.step_count == s.step_count == steps
        xb = b.current_state.particle_positions.cpu().numpy()
        xs = s.current_state.particle_positions.cpu().numpy()
        dx = sc.simulation.grid_spacing
        np.testing.assert_allclose(xb, xs, rtol=0, atol=1e-4 * dx)
        tb, ts = b.current_state.transport_state, s.current_state.transport_state
        Tb = tb.temperatures.cpu().numpy()
        np.testing.assert_allclose(Tb, ts.temperatures.cpu().numpy(), rtol=1e-6)
        assert Tb.max() > sc.transport.initial_temperature_k   # the oven is heating each body
        for name in ("water_masses", "heat_exchanges", "water_losses"):
            np.testing.assert_allclose(getattr(tb, name).cpu().numpy(), getattr(ts, name).cpu().numpy(),
                                       rtol=1e-5, atol=1e-12, err_msg=name)
        np.testing.assert_allclose(b.current_state.material_state.porosities.cpu().numpy(),
                                   s.current_state.material_state.porosities.cpu().numpy(), rtol=0,
                                   atol=porosity_atol)


@pytest.mark.parametrize("launch,groups,table_particles",
                         [("table", 2, 0), ("table", 1, 0), ("streams", 1, 0), ("auto", 2, 12_000)])
@pytest.mark.parametrize("prestrain", [(0.0, 0.0), (0.04, 0.1)])
def test_graph_replay_matches_individual_advance(prestrain, launch, groups, table_particles):
    from baking_b200 import scenes
    from baking_b200.batch import BatchedSimulators
    scs = bodies(prestrain)
    batched = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    single = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    batch = BatchedSimulators(batched, streams=4, launch=launch, groups=groups, table_particles=table_particles)
    if launch == "auto":  # bodies of 5k-20k particles: some through a table, some on their own
        assert batch.table_sims and batch.stream_sims
    batch.capture()   # capture runs two substeps
    batch.Advance(10)
    for sim in single:
        sim.AdvanceUnchecked(12)
    _compare(batched, single, scs, 12)
    for st in batch.CheckState():
        assert st["step_count"] == 12


def test_instance_table_without_graph_and_after_outside_steps():
    """The table launch stepped eagerly (graph=False), then after one substep taken outside the
    batch (which swaps every ping-pong pair, so the table is rebuilt), against the bodies advanced
    one by one; the per-stage launches each cover the whole batch."""
    from baking_b200 import _lib, scenes
    from baking_b200.batch import BatchedSimulators
    scs = bodies((0.04, 0.1))
    batched = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    single = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    batch = BatchedSimulators(batched, launch="table", groups=1)
    timer = _lib.KernelTimer()
    with timer:
        batch.Advance(4, graph=False)
    kernels = timer.summary()
    assert kernels["batch_p2g"]["count"] == 4 and kernels["batch_g2p_return"]["count"] == 4
    assert kernels["batch_transport_scatter"]["count"] == 2   # the second of each pair is scattered ahead
    assert "p2g" not in kernels
    for sim in batched:
        sim.AdvanceUnchecked(1)
    batch.Advance(4)   # rebuilds the table and captures (two substeps), then replays twice
    for sim in single:
        sim.AdvanceUnchecked(11)
    _compare(batched, single, scs, 11)


def test_instance_table_with_surrogate_on_some_instances():
    """Instances with the learned return map take the surrogate G2P kernel, the others the exact
    one, in the same batched substep; each matches its body advanced alone."""
    from baking_b200 import scenes
    from baking_b200.batch import BatchedSimulators
    from baking_b200.surrogate import LoadReturnSurrogate, ReturnMapSurrogate
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    net = LoadReturnSurrogate(root / "baking_b200" / "data" / "return_surrogate_box_loaf.npz")
    scs = bodies((0.04, 0.1))
    batched = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    single = [scenes.make_simulator(s, diagnostics="lean") for s in scs]
    for k in (0, 2, 4):
        ReturnMapSurrogate(net).attach(batched[k])
        ReturnMapSurrogate(net).attach(single[k])
    BatchedSimulators(batched, launch="table").Advance(6)   # capture runs two substeps first
    for sim in single:
        sim.AdvanceUnchecked(8)
    # float summation order differs between the launches; the network passes those differences on
    _compare(batched, single, scs, 8, porosity_atol=1e-5)


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


def test_substep_graphs_match_eager_steps_and_step_summary():
    """SubstepGraphs (one graph launch per substep, with the step-result reduction) against the
    same body stepped eagerly; StepSummary against its definition computed with torch."""
    import torch
    from baking_b200 import scenes
    from baking_b200.batch import SubstepGraphs
    sc = scenes.dough_ball(48, 20_000, seed=5, prestrain=0.05)
    graphed = scenes.make_simulator(sc, diagnostics="lean")
    eager = scenes.make_simulator(sc, diagnostics="lean")
    stepper = SubstepGraphs(graphed).capture()  # runs two substeps
    for _ in range(7):
        result = stepper.Advance(1).cpu().numpy()
    eager.AdvanceUnchecked(9)
    assert graphed.step_count == eager.step_count == 9
    dx = sc.simulation.grid_spacing
    np.testing.assert_allclose(graphed.current_state.particle_positions.cpu().numpy(),
                               eager.current_state.particle_positions.cpu().numpy(), rtol=0, atol=1e-4 * dx)
    masses = graphed.Masses().double()
    v = graphed.current_state.particle_velocities.double()
    expected = [float(graphed.grid_state.node_masses.double().sum()), float(0.5 * (masses * (v * v).sum(1)).sum())]
    # the particle masses of Masses() are float32: 1e-6
    np.testing.assert_allclose(result, expected, rtol=1e-6)
    np.testing.assert_allclose(graphed.StepSummary().cpu().numpy(), expected, rtol=1e-6)
    del stepper
    torch.cuda.synchronize()


def test_substep_graphs_staged_inputs():
    """Inputs uploaded with load() on a copy stream are the ones the next substep uses."""
    import torch
    from baking_b200 import scenes
    from baking_b200.batch import SubstepGraphs
    sc = scenes.dough_ball(32, 8_000, seed=2)
    sim = scenes.make_simulator(sc, diagnostics="lean")
    rates = sim.material.production_parameter
    stepper = SubstepGraphs(sim, inputs=[rates]).capture()
    copy = torch.cuda.Stream()
    zero = torch.zeros(rates.shape, dtype=rates.dtype).pin_memory()
    some = torch.full(rates.shape, 1e-3, dtype=rates.dtype).pin_memory()
    stepper.load([zero], 0, copy)
    stepper.load([some], 1, copy)
    n0 = sim.current_state.material_state.gas_moles.clone()
    stepper.Advance(1)
    n1 = sim.current_state.material_state.gas_moles.clone()
    assert torch.equal(n0, n1)          # no source in the substep that read the zero rates
    stepper.Advance(1)
    assert bool((sim.current_state.material_state.gas_moles > n1).all())
    torch.testing.assert_close(rates, some.to(rates.device))
    del stepper
    torch.cuda.synchronize()


def test_substep_graphs_host_results():
    """Results written by the graphs into mapped host memory match StepSummary, substep by substep,
    read one substep behind while the next one runs."""
    import torch
    from baking_b200 import scenes
    from baking_b200.batch import SubstepGraphs
    sc = scenes.dough_ball(32, 8_000, seed=4)
    sim = scenes.make_simulator(sc, diagnostics="lean")
    stepper = SubstepGraphs(sim, host_results=True).capture()
    pending, got, expected = None, [], []
    for _ in range(4):
        step = stepper.Advance(1)
        torch.cuda.current_stream().synchronize()
        expected.append(sim.StepSummary().cpu().numpy().tolist())
        if pending is not None:
            got.append(pending.get())
        pending = step
    got.append(pending.get())
    np.testing.assert_allclose(np.array(got), np.array(expected), rtol=1e-12)
    del stepper
    torch.cuda.synchronize()


def test_chained_substep_graphs_match_eager_steps():
    """SubstepGraphs(chained=True): every graph scatters the next substep's transport fields ahead and
    uses the ones the previous substep scattered. Stepping the simulator outside the object in
    between makes the next substep scatter its own fields. Both match eager stepping; a state
    array given as an input is refused."""
    import pytest
    import torch
    from baking_b200 import scenes
    from baking_b200.batch import SubstepGraphs
    sc = scenes.dough_ball(48, 20_000, seed=6, prestrain=0.05)
    graphed = scenes.make_simulator(sc, diagnostics="lean")
    eager = scenes.make_simulator(sc, diagnostics="lean")
    with pytest.raises(ValueError):
        SubstepGraphs(graphed, inputs=[graphed.current_state.transport_state.temperatures], chained=True)
    stepper = SubstepGraphs(graphed, inputs=[graphed.material.production_parameter], chained=True).capture()
    assert stepper.chained
    stepper.Advance(5)
    graphed.AdvanceUnchecked(3)   # outside the object: the next graph substep resynchronises
    stepper.Advance(4)
    for _ in range(14):
        eager.Step()
    assert graphed.step_count == eager.step_count == 14
    dx = sc.simulation.grid_spacing
    np.testing.assert_allclose(graphed.current_state.particle_positions.cpu().numpy(),
                               eager.current_state.particle_positions.cpu().numpy(), rtol=0, atol=1e-4 * dx)
    np.testing.assert_allclose(graphed.current_state.transport_state.temperatures.cpu().numpy(),
                               eager.current_state.transport_state.temperatures.cpu().numpy(), rtol=1e-9)
    del stepper
    torch.cuda.synchronize()
