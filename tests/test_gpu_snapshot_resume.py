"""Resuming from a snapshot (MpmSimulator.LoadSnapshot; the reference writes snapshots with
physics/mpm.py:310-340 but cannot load them): a run saved after k substeps and resumed in a new
simulator continues as the uninterrupted run, through the settling-to-baking switch, with a sorted
particle order, and snapshots of another scene are refused."""
from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host(t):
    from baking_b200 import arrays
    return arrays.to_numpy(t)


def _same_state(a, b):
    sa, sb = a.current_state, b.current_state
    # float atomics may sum in another order between the two runs
    for name, atol in (("particle_positions", 1e-6), ("particle_velocities", 1e-5), ("deformation_gradients", 1e-5)):
        np.testing.assert_allclose(_host(getattr(sb, name)), _host(getattr(sa, name)), rtol=0, atol=atol, err_msg=name)
    ma, mb = sa.material_state, sb.material_state
    np.testing.assert_allclose(_host(mb.porosities), _host(ma.porosities), rtol=1e-5, atol=1e-7)
    np.testing.assert_array_equal(_host(mb.gelled), _host(ma.gelled))
    ta, tb = sa.transport_state, sb.transport_state
    np.testing.assert_allclose(_host(tb.temperatures), _host(ta.temperatures), rtol=1e-9)
    np.testing.assert_allclose(_host(tb.water_masses), _host(ta.water_masses), rtol=1e-7)
    np.testing.assert_allclose(_host(tb.heat_exchanges), _host(ta.heat_exchanges), rtol=1e-7, atol=1e-15)
    np.testing.assert_allclose(_host(mb.gas_moles), _host(ma.gas_moles), rtol=1e-7)
    assert a.step_count == b.step_count and a.baking_time == b.baking_time
    assert a.IsSettling == b.IsSettling and a.settling_reason == b.settling_reason


def test_resume_continues_the_run(tmp_path):
    from baking_b200.scenes import dough_ball, make_simulator
    scene = dough_ball(32, 4000, seed=4, initial_temperature=330.0)
    a = make_simulator(scene)
    a.Advance(5)
    path = tmp_path / "snapshot.npz"
    a.SaveSnapshot(path)
    a.Advance(5)
    b = make_simulator(scene)
    b.Advance(2)  # loading replaces whatever state the simulator had
    b.LoadSnapshot(path)
    assert b.step_count == 5
    np.testing.assert_array_equal(_host(b.vertex_positions), np.load(path)["vertices"])
    b.Advance(5)
    _same_state(a, b)


def test_resume_across_the_settling_switch(tmp_path):
    from baking_b200.config import TransportConfig
    from tests.scenes import build_transport
    config = TransportConfig(enabled=True, settling_duration_s=0.0004)
    a = build_transport("cuda", config, gas=True)
    a.Advance(2)
    assert a.IsSettling
    snap = a.CaptureSnapshot()
    a.Advance(4)
    assert not a.IsSettling and a.baking_steps == 2
    b = build_transport("cuda", config, gas=True)
    b.LoadSnapshot(snap)
    assert b.IsSettling and b.step_count == 2
    b.Advance(4)
    _same_state(a, b)


def test_resume_a_sorted_run(tmp_path):
    from baking_b200.scenes import dough_ball, make_simulator, permuted
    scene = dough_ball(32, 4000, seed=6, initial_temperature=330.0)
    scene = permuted(scene, np.random.default_rng(1).permutation(len(scene.samples.particle_positions)))
    a = make_simulator(scene)
    a.SortParticles()
    a.Advance(3)
    path = tmp_path / "sorted.npz"
    a.SaveSnapshot(path)
    a.Advance(3)
    b = make_simulator(scene)
    b.LoadSnapshot(path)
    np.testing.assert_array_equal(b.particle_order.cpu().numpy(), a.particle_order.cpu().numpy())
    b.Advance(3)
    _same_state(a, b)


def test_snapshot_of_another_scene_is_refused(tmp_path):
    from baking_b200.scenes import dough_ball, make_simulator
    a = make_simulator(dough_ball(32, 4000, seed=4))
    snap = a.CaptureSnapshot()
    other = make_simulator(dough_ball(32, 12000, seed=4))
    assert other.particle_data.particle_count != a.particle_data.particle_count
    with pytest.raises(ValueError):
        other.LoadSnapshot(snap)
    legacy = {k: v for k, v in snap.items() if not k.startswith("resume_")}
    with pytest.raises(ValueError, match="resume"):
        make_simulator(dough_ball(32, 4000, seed=4)).LoadSnapshot(legacy)
