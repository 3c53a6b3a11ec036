"""Hand-written adjoint of the mechanics substep against finite differences and the reference's
autodiff known answers (tests/test_warp_autodiff.py:27-58, tests/test_ding.py:140-171). The
transport substep's adjoint is checked in test_gpu_adjoint_transport.py with the same helpers.

Every gradient is checked as a directional derivative: <dL/dtheta, delta> against the central
difference (L(theta + eps delta) - L(theta - eps delta)) / (2 eps) of the float32 forward run.
"""
from dataclasses import replace

import numpy as np
import pytest

from baking_b200.config import DingConfig, MaterialConfig, SimulationConfig
from baking_b200.geometry import CreateDemoMesh, SampleParticles

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def velocity_sim():
    from baking_b200.physics.mpm import MpmSimulator
    mesh = CreateDemoMesh(1)
    return MpmSimulator(mesh, SampleParticles(mesh, 1000.0, 4),
                        replace(SimulationConfig(), grid_resolution=20, grid_spacing=0.05, time_step=0.001,
                                gravity=(0.0, 0.0, 0.0), device_name="cuda:0"),
                        MaterialConfig())


def velocity_loss(value, grad):
    """tests/test_warp_autodiff.py:27-49: v = (value, 0, 0), 3 substeps, mean x displacement."""
    torch = _torch()
    from baking_b200.physics.adjoint import Rollout
    sim = velocity_sim()
    x0 = sim.current_state.particle_positions.clone()
    param = torch.tensor([value], dtype=torch.float32, device="cuda", requires_grad=grad)
    v = param * torch.tensor([1.0, 0.0, 0.0], device="cuda")
    out = Rollout(sim, 3, velocities=v.expand(x0.shape[0], 3))
    loss = (out["positions"][:, 0] - x0[:, 0]).mean()
    if grad:
        loss.backward()
        return float(loss.detach()), float(param.grad[0])
    return float(loss.detach()), None


def test_velocity_gradient_known_answer():
    _, gradient = velocity_loss(0.2, True)
    fd = (velocity_loss(0.3, False)[0] - velocity_loss(0.1, False)[0]) / 0.2
    np.testing.assert_allclose(gradient, fd, rtol=0.01, atol=1e-6)
    np.testing.assert_allclose(gradient, 0.003, rtol=0.01, atol=1e-6)


STRAIN_RATES = np.diag([1.5, -0.75, 0.2]).astype(np.float32)


def ding_sim(viscosity, ding=None, material=None, mesh_subdivisions=1, time_step=0.001):
    from baking_b200.physics.mpm import MpmSimulator
    from tests.scenes import assign, to_np
    mesh = CreateDemoMesh(mesh_subdivisions)
    sim = MpmSimulator(mesh, SampleParticles(mesh, 1000.0, 4),
                       replace(SimulationConfig(), device_name="cuda:0", time_step=time_step,
                               gravity=(0.0, 0.0, 0.0)),
                       material or MaterialConfig(model="ding2019"),
                       ding_config=ding or DingConfig(yield_stress=5.0, viscosity=viscosity))
    st = sim.current_state
    x = to_np(st.particle_positions)
    assign(st.particle_velocities, ((x - np.array([0.5, 0.6, 0.5], np.float32)) @ STRAIN_RATES.T).astype(np.float32))
    assign(st.affine_velocities, np.tile(STRAIN_RATES, (len(x), 1, 1)))
    return sim


def ding_viscosity_loss(value, grad):
    """tests/test_ding.py:140-161: 5 substeps, loss = mean tau_00 of the final state."""
    torch = _torch()
    from baking_b200.physics.adjoint import Rollout
    sim = ding_sim(value)
    eta = torch.tensor([value], dtype=torch.float32, device="cuda", requires_grad=grad)
    out = Rollout(sim, 5, checkpoint_every=2, viscosity_parameter=eta)
    loss = out["kirchhoff_stresses"][:, 0, 0].mean()
    sim.CheckState()
    if grad:
        loss.backward()
        return float(loss.detach()), float(eta.grad[0])
    return float(loss.detach()), None


def test_ding_mpm_viscosity_gradient_known_answer():
    _, gradient = ding_viscosity_loss(1000.0, True)
    fd = (ding_viscosity_loss(1010.0, False)[0] - ding_viscosity_loss(990.0, False)[0]) / 20.0
    assert abs(fd) > 1e-7
    np.testing.assert_allclose(gradient, fd, rtol=0.03, atol=1e-7)


# ----------------------------------------------------------------- directional checks
def _coherent(shape, seed, spread=0.25):
    """Random values shared by every particle plus a smaller per-particle part. Against a loss of the
    same form the signal adds up over particles while float32 rounding of the forward run does not."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    common = torch.randn((1,) + tuple(shape[1:]), generator=g, dtype=torch.float64)
    return (common + spread * torch.randn(tuple(shape), generator=g, dtype=torch.float64)).to("cuda")


def _weights(shapes, seed):
    return {k: _coherent(s, seed + i) for i, (k, s) in enumerate(shapes.items())}


def directional_check(make_sim, steps, name, delta, eps, checkpoint_every=2, rtol=1e-3):
    """Per output array k: <dL_k/d name, delta> against central differences of L_k = <W_k, out_k>.

    The tolerance is 1e-3 relative to the unsigned size of the change, sum |W_k * d out_k|, so that
    terms cancelling in L_k do not inflate it, plus two error estimates of the differences
    themselves: their change between steps eps and eps/2 (the truncation error), and the rounding
    of the outputs (float32, or float64 for the transport and gas fields). At least one output must
    be resolved to 5% of its change for the check to count."""
    torch = _torch()
    from baking_b200.physics.adjoint import Rollout

    def base_value(sim):
        st = sim.current_state
        if name == "viscosity_parameter":
            return sim.material.viscosity_parameter.clone()
        if name == "young_modulus":
            return torch.tensor([sim.material.material_config.young_modulus], dtype=torch.float32, device="cuda")
        if name == "heat_transfer_parameter":
            return sim.transport.heat_transfer_parameter.clone()
        if name == "gas_source_rates":
            return sim.material.production_parameter.clone()
        attr = {"positions": "particle_positions", "velocities": "particle_velocities",
                "affine_velocities": "affine_velocities", "deformation_gradients": "deformation_gradients"}
        if name in attr:
            return getattr(st, attr[name]).clone()
        transport = {"transport_temperatures": "temperatures", "water_masses": "water_masses"}
        if name in transport:
            return getattr(st.transport_state, transport[name]).clone()
        return getattr(st.material_state, name).clone()

    def run(scale, grad):
        sim = make_sim()
        theta = base_value(sim)
        param = (theta.double() + scale * delta.double()).to(theta.dtype).detach().requires_grad_(grad)
        return param, Rollout(sim, steps, checkpoint_every=checkpoint_every, **{name: param})

    _, out0 = run(0.0, False)
    weights = _weights({k: tuple(v.shape) for k, v in out0.items()}, 7)

    def diff(h):
        plus, minus = run(h, False)[1], run(-h, False)[1]
        return {k: (plus[k].double() - minus[k].double()) / (2 * h) for k in plus}

    d1, d2 = diff(eps), diff(eps / 2)
    resolved = []
    for k in out0:
        w = weights[k]
        fd1, fd2 = float((w * d1[k]).sum()), float((w * d2[k]).sum())
        size = float((w * d2[k]).abs().sum())
        ulp = 2.0 ** -52 if out0[k].dtype == torch.float64 else 2.0 ** -23
        rounding = float((w.abs() * out0[k].double().abs()).sum()) * ulp / (eps / 2)
        param, out = run(0.0, True)
        (out[k].double() * w).sum().backward()
        analytic = float((param.grad.double() * delta.double()).sum())
        if max(abs(analytic), size) < 1e-12:
            continue  # this output does not depend on the input
        spread = abs(fd1 - fd2)
        assert abs(analytic - fd2) <= rtol * size + 2 * spread + 2 * rounding, \
            f"{name} -> {k}: adjoint {analytic} vs FD {fd2} (FD at 2h {fd1}, size {size}, rounding {rounding})"
        if spread + rounding < 0.05 * size and abs(analytic - fd2) <= 0.05 * size:
            resolved.append(k)
    assert resolved, f"{name}: no output resolved by the finite differences"


def neo_hookean_sim():
    from baking_b200.physics.mpm import MpmSimulator
    from tests.scenes import assign, to_np
    mesh = CreateDemoMesh(2)
    sim = MpmSimulator(mesh, SampleParticles(mesh, 1000.0, 4),
                       replace(SimulationConfig(), device_name="cuda:0", time_step=0.001, gravity=(0.0, -9.81, 0.0)),
                       MaterialConfig(young_modulus=20000.0))
    st = sim.current_state
    x = to_np(st.particle_positions)
    rng = np.random.default_rng(3)
    rates = STRAIN_RATES + 0.3 * rng.standard_normal((3, 3)).astype(np.float32)
    assign(st.particle_velocities, ((x - np.array([0.5, 0.6, 0.5], np.float32)) @ rates.T).astype(np.float32))
    assign(st.affine_velocities, np.tile(rates, (len(x), 1, 1)))
    F = np.eye(3, dtype=np.float32) + 0.05 * rng.standard_normal((len(x), 3, 3)).astype(np.float32)
    assign(st.deformation_gradients, F)
    return sim


def _delta(shape, seed, scale=1.0):
    return scale * _coherent(shape, seed)


@pytest.mark.parametrize("name,scale,eps", [
    ("velocities", 0.05, 0.5), ("positions", 0.002, 0.5), ("affine_velocities", 0.5, 0.5),
    ("deformation_gradients", 0.01, 0.5), ("young_modulus", 1000.0, 0.5)])
def test_neo_hookean_directional(name, scale, eps):
    sim = neo_hookean_sim()
    n = sim.particle_data.particle_count
    shape = {"velocities": (n, 3), "positions": (n, 3), "affine_velocities": (n, 3, 3),
             "deformation_gradients": (n, 3, 3), "young_modulus": (1,)}[name]
    directional_check(neo_hookean_sim, 6, name, _delta(shape, 11, scale), eps, checkpoint_every=4)


def porous_ding_sim(temperature=False, porosity=0.3):
    # Yield stress 50 Pa: float32 Hencky stresses carry ~1e-3 Pa of rounding at E = 2e4 Pa, which
    # must stay well below the stress changes the finite differences resolve.
    ding = DingConfig(yield_stress=50.0, viscosity=1000.0, porosity=porosity, temperature_enabled=temperature)
    sim = ding_sim(1000.0, ding=ding, mesh_subdivisions=2)
    from tests.scenes import assign
    rng = np.random.default_rng(5)
    n = sim.particle_data.particle_count
    st = sim.current_state
    Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    Q *= np.sign(np.linalg.det(Q))
    Fe = (Q @ np.diag([1.01, 0.995, 1.003]) @ Q.T)[None] + 0.003 * rng.standard_normal((n, 3, 3))
    assign(st.material_state.elastic_gradients, Fe.astype(np.float32))
    assign(st.deformation_gradients, Fe.astype(np.float32))
    tau = 20.0 * rng.standard_normal((n, 3, 3))
    assign(st.material_state.kirchhoff_stresses, (tau + tau.transpose(0, 2, 1)).astype(np.float32))
    if temperature:
        assign(st.material_state.temperatures, (300.0 + 5.0 * rng.random(n)).astype(np.float32))
    return sim


@pytest.mark.parametrize("name,scale,eps", [
    ("velocities", 0.02, 0.5), ("affine_velocities", 0.3, 0.5), ("elastic_gradients", 0.002, 0.5),
    ("kirchhoff_stresses", 5.0, 0.5), ("porosities", 0.02, 0.5), ("viscosity_parameter", 100.0, 0.5),
    ("young_modulus", 1000.0, 1.0)])
def test_porous_ding_directional(name, scale, eps):
    sim = porous_ding_sim()
    n = sim.particle_data.particle_count
    shape = {"velocities": (n, 3), "affine_velocities": (n, 3, 3), "elastic_gradients": (n, 3, 3),
             "kirchhoff_stresses": (n, 3, 3), "porosities": (n,), "viscosity_parameter": (1,),
             "young_modulus": (1,)}[name]
    directional_check(porous_ding_sim, 5, name, _delta(shape, 13, scale), eps)


@pytest.mark.parametrize("name,scale,eps", [("elastic_gradients", 0.002, 0.5), ("velocities", 0.02, 0.5)])
def test_von_mises_ding_directional(name, scale, eps):
    """Zero porosity: the isochoric correction of the return map (ding.py:129-131)."""
    make = lambda: porous_ding_sim(porosity=0.0)  # noqa: E731
    n = make().particle_data.particle_count
    shape = {"velocities": (n, 3), "elastic_gradients": (n, 3, 3)}[name]
    directional_check(make, 5, name, _delta(shape, 17, scale), eps)


def test_temperature_directional():
    make = lambda: porous_ding_sim(temperature=True)  # noqa: E731
    n = make().particle_data.particle_count
    directional_check(make, 5, "temperatures", _delta((n,), 19, 2.0), 0.5)


def test_rollout_rejects_unknown_inputs():
    from baking_b200.physics.adjoint import Rollout
    with pytest.raises(TypeError):
        Rollout(velocity_sim(), 1, gravity=1.0)
    with pytest.raises(ValueError):
        Rollout(velocity_sim(), 1, gas_source_rates=_torch().ones(1, device="cuda"))


def test_checkpoint_interval_does_not_change_gradients():
    """Recomputation only reorders float atomics, so gradients agree to float32 rounding."""
    torch = _torch()
    from baking_b200.physics.adjoint import Rollout
    grads = []
    for every in (1, 3, 16):
        sim = porous_ding_sim()
        v = sim.current_state.particle_velocities.clone().requires_grad_(True)
        out = Rollout(sim, 7, checkpoint_every=every, velocities=v)
        out["kirchhoff_stresses"][:, 0, 1].sum().backward()
        grads.append(v.grad.clone())
    scale = float(grads[0].abs().max())
    torch.testing.assert_close(grads[0], grads[1], rtol=1e-3, atol=1e-4 * scale)
    torch.testing.assert_close(grads[0], grads[2], rtol=1e-3, atol=1e-4 * scale)
