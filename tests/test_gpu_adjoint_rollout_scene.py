"""The differentiable-rollout workload at its own size, adjoint against central finite differences.

Scene: a 100,000-particle dough sphere on a 64^3 grid (the box loaf's dough: Ding with temperature
tables, porosity 0.2, gas with per-particle source rates, thermal-water transport), 64 substeps
with a checkpoint every 8. Loss: the mean squared distance of the final positions to the initial
cloud scaled by 1.2 about its centre. Inputs: the per-particle initial temperatures, the
per-particle gas source rates and Young's modulus E, perturbed by 1e-3 of their values.

So that every input moves the loss by more than the float32 forward's rounding, the sphere starts
near the gas reaction peak (330 K, where the source term exp(-((T - 333.15)/15)^2) is steep in T),
its per-particle gas source rates are drawn from [0, 0.05] (the benchmark loaf's [0, 1e-3] builds
too little pressure in 64 substeps to be resolved), and it starts with an elastic log strain of
(0.015, -0.04, 0.005), a compression with a shear part, so that its elastic rebound towards the
1.2-scaled target depends on E.

The bar: the adjoint's directional derivative agrees with the central difference to 1e-3 of its
size, plus the differences' own error estimates (their change between perturbations h and h/2,
and the rounding of the float32 positions). At least three of the four directions must be resolved
by the differences to 5%, so the check cannot pass vacuously. The reference pins the same kind of gradient on small scenes
(tests/test_warp_autodiff.py:54-61, tests/test_ding.py:105-113, tests/test_gas.py:153-160).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS, EVERY, EPS = 64, 8, 1e-3


@pytest.fixture(scope="module")
def scene():
    from dataclasses import replace
    from baking_b200.scenes import dough_ball
    base = dough_ball(64, 100_000, seed=0, initial_temperature=330.0, gas_rate_max=0.05)
    return replace(base, initial_log_strain=(0.015, -0.04, 0.005))


def _loss(scene, T_delta=None, rate_delta=None, E_scale=1.0, grad=False):
    """Loss of one rollout, and with ``grad`` the gradients (dL/dT0, dL/drates, dL/dE)."""
    import torch
    from baking_b200.physics.adjoint import Rollout
    from baking_b200.scenes import make_simulator
    sim = make_simulator(scene, diagnostics="lean")
    st = sim.current_state
    x0 = st.particle_positions.double().clone()
    center = x0.mean(0)
    target = 1.2 * (x0 - center) + center
    T0 = st.transport_state.temperatures.clone()
    rates = sim.material.production_parameter.clone()
    E0 = torch.tensor([sim.material.material_config.young_modulus * E_scale], dtype=torch.float32, device="cuda")
    if T_delta is not None:
        T0 = T0 + T_delta
    if rate_delta is not None:
        rates = (rates.double() + rate_delta).float()
    for t in (T0, rates, E0):
        t.requires_grad_(grad)
    out = Rollout(sim, STEPS, checkpoint_every=EVERY, transport_temperatures=T0, gas_source_rates=rates,
                  young_modulus=E0)
    x = out["positions"].double()
    loss = ((x - target) ** 2).sum(1).mean()
    sim.CheckState()
    # Float32 rounding of the positions moves each particle's squared distance by about
    # 2 |x - target| |x| 2^-24 per axis, independently across particles: the loss's rounding is
    # their root sum of squares over n (three standard deviations kept).
    per = 2.0 * 2.0 ** -24 * (x - target).abs() * x.abs()
    rounding = float(3.0 * per.pow(2).sum().sqrt().detach()) / x.shape[0]
    if not grad:
        return float(loss.detach()), rounding, None
    loss.backward()
    return float(loss.detach()), rounding, (T0.grad.double(), rates.grad.double(), E0.grad.double())


def _check(scene, grads, name, **delta):
    """<grad, delta> against (L(+delta) - L(-delta)) / 2 with the step halved for an error estimate."""
    def fd(h):
        kw_p = {k: (v * h if k != "E_scale" else 1.0 + (v - 1.0) * h) for k, v in delta.items()}
        kw_m = {k: (-v * h if k != "E_scale" else 1.0 - (v - 1.0) * h) for k, v in delta.items()}
        lp, rp, _ = _loss(scene, **kw_p)
        lm, rm, _ = _loss(scene, **kw_m)
        return (lp - lm) / (2.0 * h), max(rp, rm) / (2.0 * h)

    f1, r1 = fd(1.0)
    f2, r2 = fd(0.5)
    gT, gR, gE = grads
    analytic = 0.0
    if "T_delta" in delta:
        analytic += float((gT * delta["T_delta"].double()).sum())
    if "rate_delta" in delta:
        analytic += float((gR * delta["rate_delta"].double()).sum())
    if "E_scale" in delta:
        E = scene.material.young_modulus
        analytic += float(gE.sum()) * E * (delta["E_scale"] - 1.0)
    spread = abs(f1 - f2)
    size = abs(f2)
    print(f"\n[{name}] adjoint {analytic:.6e}  FD(h) {f1:.6e}  FD(h/2) {f2:.6e}  rounding {r2:.2e}")
    assert abs(analytic - f2) <= 1e-3 * size + 2 * spread + 2 * r2, \
        f"{name}: adjoint {analytic} vs finite difference {f2} (at 2h {f1})"
    return spread + r2 < 0.05 * size


def test_rollout_gradients_against_finite_differences(scene):
    import torch
    _, _, grads = _loss(scene, grad=True)
    n = scene.particle_count
    assert all(bool(torch.isfinite(g).all()) for g in grads)
    T = 330.0
    rates = torch.as_tensor(scene.gas_source_rates, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(3)
    signs = torch.as_tensor(rng.choice([-1.0, 1.0], n), device="cuda")
    resolved = [
        _check(scene, grads, "T0 uniform", T_delta=torch.full((n,), EPS * T, dtype=torch.float64, device="cuda")),
        _check(scene, grads, "T0 random signs", T_delta=EPS * T * signs),
        _check(scene, grads, "gas source rates", rate_delta=EPS * rates),
        _check(scene, grads, "E", E_scale=1.0 + EPS)]
    # The random-sign direction cancels most of the per-particle terms; the coherent ones must resolve.
    assert sum(resolved) >= 3, f"only {sum(resolved)} of 4 directions resolved by the differences"
