"""Reordering particles by grid cell on the device: bk_sort_by_cell against a numpy restatement
of its keys (float32 stencil bases, Morton interleave, stable order, particles whose stencil
leaves the grid last), and MpmSimulator.SortParticles on a shuffled dough sphere against the same
scene run unsorted (positions, temperatures, gas, mesh vertices), its renumbered mesh binding and
face owners, Reset after a sort and the recorder's regions."""
from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def numpy_cell_order(x, origin, dx, R):
    g = (x.astype(np.float32) - np.asarray(origin, np.float32)) / np.float32(dx)
    with np.errstate(invalid="ignore"):
        b = np.where(np.isfinite(g), np.floor(g - np.float32(0.5)), -1.0).astype(np.int64)
    valid = np.isfinite(x).all(axis=1) & (b >= 0).all(axis=1) & (b + 2 < R).all(axis=1)
    bits = max(1, (R - 1).bit_length())

    def spread(v):
        out = np.zeros(len(v), dtype=np.uint64)
        for k in range(21):
            out |= ((v >> k) & 1).astype(np.uint64) << np.uint64(3 * k)
        return out

    key = spread(b[:, 2]) | (spread(b[:, 1]) << np.uint64(1)) | (spread(b[:, 0]) << np.uint64(2))
    key[~valid] = np.uint64((1 << (3 * bits)) - 1)
    return np.argsort(key, kind="stable")


def device_cell_order(x, origin, dx, R):
    import ctypes
    import torch
    from baking_b200 import _lib, arrays
    dev = torch.device("cuda:0")
    n = len(x)
    xd = arrays.from_numpy(x.astype(np.float32), "f4", dev) if n else arrays.vec3s(0, device=dev)
    lib = _lib.load()
    need = lib.bk_sort_by_cell_scratch_bytes(n, R)
    assert need >= 0
    scratch = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
    order = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    o = (ctypes.c_float * 3)(*origin)
    _lib.call("bk_sort_by_cell", n, arrays.layout_pitch(xd) if n else 0, arrays.ptr(xd), ctypes.addressof(o), dx, R,
              order.data_ptr(), scratch.data_ptr(), need, _lib.stream_handle())
    torch.cuda.synchronize()
    return order[:n].cpu().numpy()


@pytest.mark.parametrize("n,R", [(0, 16), (1, 16), (257, 16), (5000, 100), (40000, 128)])
def test_cell_order_matches_numpy(n, R):
    rng = np.random.default_rng(n + R)
    dx = 1.0 / R
    x = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    if n > 10:
        x[:n // 10] = x[0]          # many particles in one cell: stability
        x[n // 10: n // 10 + 5] = [[-0.2, 0.5, 0.5], [0.5, 1.3, 0.5], [0.5, 0.5, 0.999],
                                   [0.0, 0.0, 0.0], [np.nan, 0.5, 0.5]][: min(5, n - n // 10)]
    got = device_cell_order(x, (0.0, 0.0, 0.0), dx, R)
    np.testing.assert_array_equal(got, numpy_cell_order(x, (0.0, 0.0, 0.0), dx, R))


def test_scratch_query_rejects_bad_arguments():
    from baking_b200 import _lib
    lib = _lib.load()
    assert lib.bk_sort_by_cell_scratch_bytes(-1, 64) == -1
    assert lib.bk_sort_by_cell_scratch_bytes(10, 2) == -1
    assert lib.bk_sort_by_cell_scratch_bytes(0, 64) == 0


def _shuffled_sphere(seed=3):
    from baking_b200.scenes import dough_ball, permuted
    scene = dough_ball(32, 6000, seed=1, initial_temperature=330.0)
    rng = np.random.default_rng(seed)
    return permuted(scene, rng.permutation(len(scene.samples.particle_positions)))


def _host(t):
    from baking_b200 import arrays
    return arrays.to_numpy(t)


def test_sorted_run_matches_unsorted_run():
    import torch
    from baking_b200.scenes import make_simulator
    scene = _shuffled_sphere()
    plain = make_simulator(scene)
    ordered = make_simulator(scene)
    order = ordered.SortParticles()
    assert ordered.sort_count == 1
    np.testing.assert_array_equal(ordered.particle_order.cpu().numpy(), order.cpu().numpy())
    # idempotent: the sorted particles are already in cell order
    assert torch.equal(ordered.CellOrder(), torch.arange(len(order), device=order.device))
    # the renumbered binding reconstructs the same mesh
    plain.UpdateMesh(force_update=True)
    ordered.UpdateMesh(force_update=True)
    np.testing.assert_array_equal(_host(ordered.vertex_positions), _host(plain.vertex_positions))
    src = order.cpu().numpy()
    assert sorted(ordered.transport.owners.cpu().numpy().tolist()) == \
        sorted(np.argsort(src)[plain.transport.owners.cpu().numpy()].tolist())
    plain.Advance(20)
    ordered.Advance(20)
    a, b = plain.current_state, ordered.current_state
    # float sums in another order only
    np.testing.assert_allclose(_host(b.particle_positions), _host(a.particle_positions)[src], rtol=0, atol=2e-6)
    np.testing.assert_allclose(_host(b.deformation_gradients), _host(a.deformation_gradients)[src], rtol=0,
                               atol=2e-5)
    ta, tb = a.transport_state, b.transport_state
    np.testing.assert_allclose(_host(tb.temperatures), _host(ta.temperatures)[src], rtol=1e-7)
    np.testing.assert_allclose(_host(tb.water_masses), _host(ta.water_masses)[src], rtol=1e-6)
    np.testing.assert_allclose(_host(tb.heat_exchanges), _host(ta.heat_exchanges)[src], rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(_host(b.material_state.gas_moles), _host(a.material_state.gas_moles)[src], rtol=1e-6)
    plain.UpdateMesh(force_update=True)
    ordered.UpdateMesh(force_update=True)
    np.testing.assert_allclose(_host(ordered.vertex_positions), _host(plain.vertex_positions), rtol=0, atol=2e-6)


def test_reset_after_sort_starts_sorted_and_snapshot_names_the_order():
    import torch
    from baking_b200.scenes import make_simulator
    sim = make_simulator(_shuffled_sphere(seed=5))
    order = sim.SortParticles().cpu().numpy()
    sim.Advance(4)
    sim.Reset()
    n = len(order)
    assert torch.equal(sim.CellOrder(), torch.arange(n, device=sim.device))
    np.testing.assert_array_equal(_host(sim.current_state.particle_positions),
                                  sim.particle_samples.particle_positions.astype(np.float32))
    snap = sim.CaptureSnapshot()
    np.testing.assert_array_equal(snap["particle_order"], order)


def test_sort_rejects_history_and_non_permutations():
    from baking_b200.scenes import dough_ball, make_simulator
    sim = make_simulator(dough_ball(32, 2000, seed=2))
    with pytest.raises(ValueError):
        sim.SortParticles(order=np.zeros(sim.particle_data.particle_count, np.int64))
    kept = make_simulator(dough_ball(32, 2000, seed=2), retain_history=True)
    with pytest.raises(ValueError):
        kept.SortParticles()


def test_recorder_regions_follow_the_order(tmp_path):
    from baking_b200.config import ExperimentConfig, RunConfig
    from baking_b200.recording import SimulationRecorder
    from baking_b200.scenes import make_simulator
    sim = make_simulator(_shuffled_sphere(seed=9))
    sim.Advance(3)
    config = replace(ExperimentConfig(), run=replace(RunConfig(), log_path=str(tmp_path)))
    rec = SimulationRecorder(sim, config)
    before = rec.Measure()
    sim.SortParticles()
    after = rec.Measure()
    for key, value in before.items():
        if key == "energy_balance_error_j":
            # energy - initial energy - heat exchanged: a difference of float64 sums over the
            # particles, which a new summation order moves at the rounding level of the sums
            scale = abs(before["thermal_energy_j"])
            assert after[key] == pytest.approx(value, abs=1e-11 * scale), key
        elif isinstance(value, float):
            assert after[key] == pytest.approx(value, rel=1e-9, abs=1e-12), key
        else:
            assert after[key] == value, key


def test_rollout_gradients_follow_the_order():
    """Reverse mode on the sorted simulator: the gradients of the unsorted run, permuted."""
    from baking_b200.physics.adjoint import Rollout
    from baking_b200.scenes import make_simulator
    scene = _shuffled_sphere(seed=11)
    results = []
    for sort in (False, True):
        sim = make_simulator(scene, diagnostics="lean")
        order = sim.SortParticles().cpu().numpy() if sort else None
        T = sim.current_state.transport_state.temperatures.clone().requires_grad_(True)
        rates = sim.material.production_parameter.clone().requires_grad_(True)
        out = Rollout(sim, 4, checkpoint_every=2, transport_temperatures=T, gas_source_rates=rates)
        loss = (out["positions"].double() ** 2).sum() + out["gas_moles"].sum()
        loss.backward()
        results.append((T.grad.cpu().numpy(), rates.grad.cpu().numpy(), order))
    (gT, gr, _), (sT, sr, order) = results
    np.testing.assert_allclose(sT, gT[order], rtol=1e-4, atol=1e-5 * np.abs(gT).max())
    np.testing.assert_allclose(sr, gr[order], rtol=1e-4, atol=1e-5 * np.abs(gr).max())


def test_permute_particles_planes_and_element_sizes():
    """bk_permute_particles on float32 planes (1, 3 and 9 planes, pitch above n), float64 and int32
    arrays against numpy indexing, with a scratch buffer of the largest array (three groups) and
    one for all arrays (one group); a scratch smaller than the largest array is refused."""
    import ctypes
    import torch
    from baking_b200 import _lib, arrays
    dev = torch.device("cuda:0")
    n = 1000
    rng = np.random.default_rng(4)
    order = rng.permutation(n)
    host = [rng.standard_normal((n, 3)).astype(np.float32), rng.standard_normal((n, 3, 3)).astype(np.float32),
            rng.standard_normal(n), rng.integers(0, 9, n).astype(np.int32)]
    dev_arrays = [arrays.from_numpy(host[0], "f4", dev), arrays.from_numpy(host[1], "f4", dev),
                  torch.as_tensor(host[2], device=dev), torch.as_tensor(host[3], device=dev)]
    assert arrays.layout_pitch(dev_arrays[0]) > n
    table = (_lib.BkParticleArray * 4)(
        _lib.BkParticleArray(dev_arrays[0].data_ptr(), arrays.layout_pitch(dev_arrays[0]), 3, 4),
        _lib.BkParticleArray(dev_arrays[1].data_ptr(), arrays.layout_pitch(dev_arrays[1]), 9, 4),
        _lib.BkParticleArray(dev_arrays[2].data_ptr(), n, 1, 8),
        _lib.BkParticleArray(dev_arrays[3].data_ptr(), n, 1, 4))
    order_d = torch.as_tensor(order, dtype=torch.int32, device=dev)
    scratch = torch.empty(9 * n * 4, dtype=torch.uint8, device=dev)
    lib = _lib.load()
    assert lib.bk_permute_particles(n, order_d.data_ptr(), 4, ctypes.addressof(table), scratch.data_ptr(),
                                    9 * n * 4 - 1, _lib.stream_handle()) != 0
    _lib.call("bk_permute_particles", n, order_d.data_ptr(), 4, ctypes.addressof(table), scratch.data_ptr(),
              9 * n * 4, _lib.stream_handle())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(arrays.to_numpy(dev_arrays[0]), host[0][order])
    np.testing.assert_array_equal(arrays.to_numpy(dev_arrays[1]), host[1][order])
    np.testing.assert_array_equal(dev_arrays[2].cpu().numpy(), host[2][order])
    np.testing.assert_array_equal(dev_arrays[3].cpu().numpy(), host[3][order])
    # again with a scratch buffer for all four arrays at once: one group, two launches
    order2 = rng.permutation(n)
    order2_d = torch.as_tensor(order2, dtype=torch.int32, device=dev)
    big = torch.empty(64 * 1024, dtype=torch.uint8, device=dev)
    _lib.call("bk_permute_particles", n, order2_d.data_ptr(), 4, ctypes.addressof(table), big.data_ptr(),
              big.numel(), _lib.stream_handle())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(arrays.to_numpy(dev_arrays[0]), host[0][order][order2])
    np.testing.assert_array_equal(arrays.to_numpy(dev_arrays[1]), host[1][order][order2])
    np.testing.assert_array_equal(dev_arrays[2].cpu().numpy(), host[2][order][order2])
    np.testing.assert_array_equal(dev_arrays[3].cpu().numpy(), host[3][order][order2])


def test_sort_interval_sorts_during_advance():
    """sort_interval=5: Advance(10) sorts twice and follows the unsorted run."""
    from baking_b200.scenes import make_simulator
    scene = _shuffled_sphere(seed=13)
    plain = make_simulator(scene)
    auto = make_simulator(scene, sort_interval=5)
    plain.Advance(10)
    auto.Advance(10)
    assert auto.sort_count == 2
    src = auto.particle_order.cpu().numpy()
    np.testing.assert_allclose(_host(auto.current_state.particle_positions),
                               _host(plain.current_state.particle_positions)[src], rtol=0, atol=2e-6)
    np.testing.assert_allclose(_host(auto.current_state.transport_state.temperatures),
                               _host(plain.current_state.transport_state.temperatures)[src], rtol=1e-7)
    with pytest.raises(ValueError):
        make_simulator(scene, sort_interval=5, retain_history=True)
