"""Device Ding return map (bk_update_ding) against the CPU oracle on random trial states.

Covers the cases the float64 SVD must get right: large rotations, large and small
stretches, exactly repeated singular values, the identity, and both the uncoupled
(porosity from det Fp) and gas-coupled (end-state porosity solve) modes.
"""
import numpy as np
import pytest
import torch

from baking_b200 import arrays
from baking_b200.config import DingConfig, MaterialConfig
from baking_b200.physics.materials.ding import AllocateDingState, UpdateDing, ding_params
from oracle import ora

pytestmark = pytest.mark.gpu


def random_rotation(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
                     np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
                     np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)


def trial_states(n, seed, big=0.3, small=0.03, rate=20.0):
    rng = np.random.default_rng(seed)
    scale = np.where(rng.random((n, 1)) < 0.2, big, small)
    stretch = np.exp(scale * rng.standard_normal((n, 3)))
    stretch[: n // 16] = 1.0                                   # identity
    stretch[n // 16: n // 8, 1] = stretch[n // 16: n // 8, 0]  # repeated pair
    stretch[n // 8: n // 6] = stretch[n // 8: n // 6, :1]      # isotropic
    R1, R2 = random_rotation(rng, n), random_rotation(rng, n)
    R1[: n // 32] = np.eye(3)
    R2[: n // 32] = np.eye(3)
    Fe = (R1 * stretch[:, None, :]) @ R2
    C = rng.standard_normal((n, 3, 3)) * rate
    F = Fe @ (np.eye(3) + 0.01 * rng.standard_normal((n, 3, 3)))
    T = rng.uniform(290.0, 360.0, n)
    return Fe.astype(np.float32), C.astype(np.float32), F.astype(np.float32), T.astype(np.float32)


@pytest.mark.parametrize("gas", [False, True])
def test_return_map_matches_oracle(gas):
    n = 4096
    # Gas mode keeps the loading inside the porosity domain (end-state porosity from ~1e-4 to ~0.96).
    Fe, C, F, T = trial_states(n, seed=11, big=0.1, small=0.01, rate=5.0) if gas else trial_states(n, seed=7)
    mc = MaterialConfig(model="ding2019")
    dc = DingConfig(yield_stress=800.0, viscosity=1e6, porosity=0.2 if gas else 0.0, temperature_enabled=True,
                    gas_enabled=gas)
    dt = 1e-3
    por = np.full(n, dc.porosity, np.float32)
    gel = np.zeros(n, np.int32)
    # oracle
    out = {k: ora.f32(n, 3, 3) for k in ("Fe", "Fp", "tau")}
    sc = {k: ora.f32(n) for k in ("res", "n", "T", "ty", "eta", "pres")}
    gel_o = ora.i32(n)
    flags_o = ora.i32(3)
    p = ora.ding_params(gas, True, mc.shear_modulus, mc.lame_lambda, dc.yield_stress, dc.porosity, dt,
                        dc.temperature_knots_k, dc.yield_factors, dc.viscosity_factors)
    ora.update_ding(Fe, por, gel, F, C, out["Fe"], out["Fp"], out["tau"], sc["res"], sc["n"], sc["T"], gel_o,
                    sc["ty"], sc["eta"], np.array([dc.viscosity], np.float32), flags_o, sc["pres"], p, T)
    # device
    dev = torch.device("cuda:0")
    old = AllocateDingState(n, dev)
    new = AllocateDingState(n, dev)
    arrays.assign(old.elastic_gradients, Fe)
    arrays.assign(old.porosities, por)
    arrays.assign(old.gelled, gel)
    F_d, C_d, T_d = arrays.from_numpy(F, "f4", dev), arrays.from_numpy(C, "f4", dev), arrays.from_numpy(T, "f4", dev)
    flags = torch.zeros(3, dtype=torch.int32, device=dev)
    UpdateDing(old, F_d, C_d, new, torch.tensor([dc.viscosity], device=dev), flags, ding_params(mc, dc, dt), T_d)
    torch.cuda.synchronize()
    assert flags.tolist() == flags_o.tolist()
    fe, tau = arrays.to_numpy(new.elastic_gradients), arrays.to_numpy(new.kirchhoff_stresses)
    np.testing.assert_allclose(fe, out["Fe"], rtol=1e-4, atol=2e-6)
    tau_scale = np.abs(out["tau"]).max(axis=(1, 2), keepdims=True) + 1.0
    np.testing.assert_allclose(tau / tau_scale, out["tau"] / tau_scale, rtol=0, atol=1e-4)
    np.testing.assert_allclose(arrays.to_numpy(new.porosities), sc["n"], rtol=1e-4, atol=2e-7)
    np.testing.assert_allclose(arrays.to_numpy(new.plastic_gradients), out["Fp"], rtol=1e-4, atol=2e-5)
    np.testing.assert_array_equal(arrays.to_numpy(new.gelled), gel_o)
    np.testing.assert_allclose(arrays.to_numpy(new.yield_stresses), sc["ty"], rtol=1e-6)
    np.testing.assert_allclose(arrays.to_numpy(new.return_residuals), sc["res"], atol=1e-5)


def test_porosity_solve_matches_reference_bisection():
    """The device end-state porosity solve against the reference's 64-step bisection (oracle)."""
    from baking_b200.physics.materials.porous_return import SolvePorosity
    rng = np.random.default_rng(0)
    n = 3000
    q = rng.uniform(0, 6, n).astype(np.float32)
    p = rng.uniform(0, 40, n).astype(np.float32)
    d = (10 ** rng.uniform(-7, 1, n)).astype(np.float32)
    h = (10 ** rng.uniform(-7, 1, n)).astype(np.float32)
    e = rng.uniform(-0.1, 0.05, n).astype(np.float32)
    n0 = 0.2
    Vp = 1 - n0 + rng.uniform(1e-7, 0.6, n)
    got, pred = SolvePorosity(q, p, d, h, e, Vp, n0)
    got, pred = got.cpu().numpy(), pred.cpu().numpy()
    ref = np.array([ora.solve_porosity(*map(float, (q[i], p[i], d[i], h[i], e[i])), float(Vp[i]), n0)
                    for i in range(n)], np.float32)
    # Same float32 porosity except where the bisection's 2^-64 absolute resolution is coarser than
    # the root itself (porosities below ~1e-12).
    np.testing.assert_allclose(got, ref, rtol=2e-7, atol=1e-15)
    assert np.all(np.abs(got.astype(np.float64) - pred) <= 1e-6)
    # near-closure case of the reference's tests/test_gas.py:208-223
    fr = 3.725290298461914e-7
    got, pred = SolvePorosity([4.115], [29.464], [0.001052], [0.003390], [-0.0230067], [1 - 0.2 + fr], 0.2)
    assert 0 < float(got[0]) < fr
    np.testing.assert_allclose(float(got[0]), float(pred[0]), atol=1e-12)


def test_porosity_solve_elastic_exit_at_the_yield_margin():
    """The elastic early exit (q + a(trial) p <= 1), decided in float32 where that is certain and
    in float64 otherwise, against the oracle's float64 test on cases placed within 2e-5 relative
    of the margin, porosities from 1e-12 to 1 - 1e-7: where the reference exits elastically the
    same float32 porosity bit for bit, elsewhere within its rounding, and the prediction at it equal
    to the oracle's."""
    from baking_b200.physics.materials.porous_return import SolvePorosity
    rng = np.random.default_rng(7)
    m = 1000
    n0 = 0.2
    por = np.concatenate([rng.uniform(1e-6, 1 - 1e-7, m), 10 ** rng.uniform(-12, -1, m),
                          1 - 10 ** rng.uniform(-7, -1, m)])
    n0f = float(np.float32(n0))  # the solver takes n0 as float32
    Vp = 1.0 - n0f + por
    trial = Vp - 1.0 + n0f  # the elastic prediction as the solver forms it
    assert np.all((trial > 0) & (trial < 1))
    lg = np.log(1.0 / trial)
    a = 9.0 / (4.0 * lg * lg * (3.5 * trial + 1.0))
    p = rng.uniform(0.0, 1.0, trial.size).astype(np.float32)
    k = np.concatenate([rng.uniform(-2e-5, 2e-5, trial.size - 200), rng.uniform(-1e-12, 1e-12, 200)])
    q = np.clip(1.0 - a * p.astype(np.float64) * (1.0 + k), 0.0, None).astype(np.float32)
    d = np.full(trial.size, 1e-3, np.float32)
    h = np.full(trial.size, 3e-3, np.float32)
    e = rng.uniform(-0.05, 0.0, trial.size).astype(np.float32)
    got, pred = SolvePorosity(q, p, d, h, e, Vp, n0)
    got, pred = got.cpu().numpy(), pred.cpu().numpy()
    args = [tuple(float(v[i]) for v in (q, p, d, h, e)) for i in range(trial.size)]
    ref = np.array([ora.solve_porosity(*args[i], float(Vp[i]), n0) for i in range(trial.size)], np.float32)
    np.testing.assert_allclose(got, ref, rtol=2e-7, atol=0)
    # Where the reference's float64 test takes the elastic exit the device returns float32(trial).
    elastic = q.astype(np.float64) + a * p.astype(np.float64) <= 1.0
    np.testing.assert_array_equal(got[elastic], trial[elastic].astype(np.float32))
    np.testing.assert_array_equal(got[elastic], ref[elastic])
    ref_pred = np.array([ora.porosity_prediction(float(got[i]), *args[i], float(Vp[i]), n0)
                         for i in range(trial.size)])
    np.testing.assert_allclose(pred, ref_pred, rtol=1e-12, atol=1e-15)
    assert elastic.sum() > trial.size // 4 and (~elastic).sum() > trial.size // 4
