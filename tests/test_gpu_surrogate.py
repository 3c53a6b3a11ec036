"""The learned return-map surrogate in the fused substep: harvested training pairs against the CPU
oracle's UpdateDing (physics/materials/ding.py:140-221 restated in oracle/), and the trained network
against the exact map it replaces -- path usage, error, trajectory and kernel time."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_loaf(prestrain=0.0, seed=1):
    from baking_b200 import scenes
    return scenes.box_loaf(resolution=64, particle_count=60_000, seed=seed, initial_temperature=318.15,
                           prestrain=prestrain)


def simulator(scene):
    from baking_b200 import scenes
    return scenes.make_simulator(scene, diagnostics="lean")


def oracle_return(rows, sim):
    """Targets of harvested rows recomputed by the oracle: UpdateDing on Fe_old = diag(exp(features)),
    C = 0, the row's temperature and porosity; the returned principal stresses give the log strains
    before the volume correction, e_k = (tau_k - mean)/(2 mu) + mean/K."""
    from oracle import ora
    mc, dc = sim.material.material_config, sim.material.ding_config
    dt = sim.simulation_config.time_step
    mu, lam = mc.shear_modulus, mc.lame_lambda
    params = ora.ding_params(int(dc.gas_enabled), int(dc.temperature_enabled), mu, lam, dc.yield_stress,
                             dc.porosity, dt, dc.temperature_knots_k, dc.yield_factors, dc.viscosity_factors)
    n = len(rows)
    Fe = np.zeros((n, 3, 3), np.float32)
    for k in range(3):
        Fe[:, k, k] = np.exp(rows[:, k])
    por = (np.exp(rows[:, 6].astype(np.float64)) - 1.0 + dc.porosity).astype(np.float32)
    z = lambda *s: np.zeros(s, np.float32)  # noqa: E731
    Fe_new, Fp_new, tau_new = z(n, 3, 3), z(n, 3, 3), z(n, 3, 3)
    res, n_new, T_out, yl, visc, pres = z(n), z(n), z(n), z(n), z(n), z(n)
    gel_new, flags = np.zeros(n, np.int32), np.zeros(3, np.int32)
    ora.update_ding(Fe, por, np.zeros(n, np.int32), Fe.copy(), z(n, 3, 3), Fe_new, Fp_new, tau_new, res, n_new,
                    T_out, gel_new, yl, visc, np.array([dc.viscosity], np.float32), flags, pres, params,
                    rows[:, 3].astype(np.float32).copy())
    cs = np.stack([tau_new[:, k, k] for k in range(3)], 1).astype(np.float64)
    cm = cs.mean(1, keepdims=True)
    e = (cs - cm) / (2 * mu) + cm / (2 * mu + 3 * lam)
    return e - rows[:, :3]


def test_harvested_pairs_match_oracle_return():
    from baking_b200.surrogate import HarvestReturnSamples, RandomizeReturnInputs
    sim = simulator(small_loaf())
    RandomizeReturnInputs(sim, seed=3)
    f, t, seen = HarvestReturnSamples(sim, 1, capacity=200_000)
    assert seen > 10_000 and f.shape[0] == min(seen, 200_000)
    f, t = f.cpu().numpy(), t.cpu().numpy()
    assert np.isfinite(f).all() and np.isfinite(t).all()
    rng = np.random.default_rng(0)
    pick = rng.choice(len(f), 400, replace=False)
    rows = f[pick].astype(np.float64)
    expected = oracle_return(rows, sim)
    np.testing.assert_allclose(t[pick], expected, rtol=1e-3, atol=3e-6)
    # the features: sorted log singular values, temperature, saturation, gas, plastic volume strain
    assert np.all(f[:, 0] >= f[:, 1]) and np.all(f[:, 1] >= f[:, 2])
    assert 295.0 <= f[:, 3].min() and f[:, 3].max() <= 345.0


WEIGHTS = "baking_b200/data/return_surrogate_box_loaf.npz"


@pytest.fixture(scope="module")
def trained():
    """The committed network, trained by ``python -m baking_b200.surrogate`` on 9.5M pairs harvested
    from the randomised 1M-particle box loaf (same material and time step as these scenes)."""
    from pathlib import Path
    from baking_b200.surrogate import LoadReturnSurrogate
    root = Path(__file__).resolve().parents[1]
    with np.load(root / WEIGHTS) as d:
        meta = {k: d[k] for k in ("samples", "validation_rms_error", "target_rms", "history")}
    return LoadReturnSurrogate(root / WEIGHTS), meta


def test_training_on_harvested_pairs():
    """The device training pipeline on freshly harvested pairs of a small loaf: the loss falls by
    two orders of magnitude and the held-out error is a few percent of the targets."""
    import torch
    from baking_b200.surrogate import BuildTrainingSet, TrainReturnSurrogate
    sim = simulator(small_loaf(seed=2))
    f, t = BuildTrainingSet(sim, rounds=8, steps=3, capacity_per_round=400_000, seed=10)
    assert f.shape[0] > 500_000
    net, history, err, rms = TrainReturnSurrogate(f, t, epochs=25, batch=4096, seed=0)
    torch.cuda.synchronize()
    assert history[-1] < 0.01 * history[0], history
    assert max(e / r for e, r in zip(err, rms)) < 0.1, (err, rms)


def run(net, steps, judge_stride=0, untrained=False):
    import torch
    from baking_b200 import _lib
    from baking_b200.surrogate import ReturnMapMlp, ReturnMapSurrogate
    sim = simulator(small_loaf(prestrain=0.08, seed=5))
    sim.AdvanceUnchecked(2)
    sur = None
    if net is not None:
        if untrained:
            net = ReturnMapMlp(net.norm)
        sur = ReturnMapSurrogate(net, judge_stride=judge_stride).attach(sim)
    timer = _lib.KernelTimer()
    with timer:
        sim.AdvanceUnchecked(steps)
        times = timer.summary()
    torch.cuda.synchronize()
    sim.CheckState()
    return sim, sur, times


def test_trained_surrogate_replaces_the_exact_return(trained):
    net, meta = trained
    assert int(meta["samples"]) > 9_000_000
    assert max(meta["validation_rms_error"] / meta["target_rms"]) < 0.02, meta
    exact, _, t_exact = run(None, 30)
    sim, sur, t_sur = run(net, 30, judge_stride=4)
    stats = sur.statistics()
    assert stats["surrogate"] > 0.95 * 30 * 60_000, stats
    assert stats["judge_max_log_strain_error"] < 3e-5, stats
    x0 = small_loaf(seed=5).samples.particle_positions
    xe = exact.current_state.particle_positions.cpu().numpy().astype(np.float64)
    xs = sim.current_state.particle_positions.cpu().numpy().astype(np.float64)
    moved = np.linalg.norm(xe - x0, axis=1).max()
    dev = np.linalg.norm(xs - xe, axis=1).max()
    assert dev < 0.05 * moved, (dev, moved)
    assert dev < 1e-3 * np.abs(xe).max()
    np.testing.assert_allclose(sim.current_state.material_state.porosities.cpu().numpy(),
                               exact.current_state.material_state.porosities.cpu().numpy(), atol=2e-4)


def test_trained_network_gains_over_untrained(trained):
    """What training buys: the judge error of the trained network is far below that of the same
    architecture with its initial weights."""
    net = trained[0]
    _, sur_t, _ = run(net, 10, judge_stride=1)
    _, sur_u, _ = run(net, 1, judge_stride=1, untrained=True)
    e_trained = sur_t.statistics()["judge_max_log_strain_error"]
    e_untrained = sur_u.statistics()["judge_max_log_strain_error"]
    assert e_trained < 0.05 * e_untrained, (e_trained, e_untrained)


def test_surrogate_substeps_beat_the_exact_map_at_full_size(trained):
    """The method with the network against the method without it, on the workload the network was
    trained for: the 1,000,000-particle box loaf on 128^3, part-baked (318 K) and pre-stressed
    (prestrain 0.08) so that every particle yields, 40 substeps from the same state. The surrogate
    substeps are faster than the exact ones, and the final positions agree to 1e-3 of the largest
    position (the relative final-position error); the deviation as a fraction of the largest
    displacement is reported. Timed with CUDA events on the stepping stream, after 3 warm-up
    substeps and without the judge."""
    import torch
    from baking_b200 import scenes
    from baking_b200.surrogate import ReturnMapSurrogate
    net = trained[0]
    loaf = scenes.box_loaf(resolution=128, particle_count=1_000_000, seed=0, initial_temperature=318.15,
                           prestrain=0.08)
    steps, out = 40, {}
    for mode in ("exact", "surrogate"):
        sim = simulator(loaf)
        sur = ReturnMapSurrogate(net).attach(sim) if mode == "surrogate" else None
        sim.AdvanceUnchecked(3)
        stream = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        sim.AdvanceUnchecked(steps)
        b.record(stream)
        torch.cuda.synchronize()
        sim.CheckState()
        out[mode] = (a.elapsed_time(b), sim.current_state.particle_positions.double().clone(),
                     sur.statistics() if sur else None)
        del sim, sur
        torch.cuda.empty_cache()
    (t_exact, xe, _), (t_sur, xs, stats) = out["exact"], out["surrogate"]
    assert stats["surrogate"] > 0.99 * steps * loaf.particle_count, stats
    x0 = torch.as_tensor(loaf.samples.particle_positions, device=xe.device)
    dev = float((xs - xe).norm(dim=1).max())
    rel = dev / float(xe.norm(dim=1).max())
    moved = float((xe - x0).norm(dim=1).max())
    info = dict(exact_ms=t_exact, surrogate_ms=t_sur, relative_position_error=rel, deviation_over_displacement=dev / moved)
    assert t_sur < t_exact, info
    assert rel < 1e-3, info
