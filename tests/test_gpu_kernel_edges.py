"""Edge cases of the transfer kernels through the C ABI (bk_particle_to_grid, bk_update_grid,
bk_grid_to_particle) against the oracle's restatement of physics/transfer.py:36-109 and
physics/grid.py:20-38: ragged particle counts around the block size (including none), particles
whose stencil leaves the grid (flagged and skipped, the others still transferred), and the wall
clamp in the boundary cells."""
from dataclasses import replace

import numpy as np
import pytest

from baking_b200.config import SimulationConfig
from oracle import ora

pytestmark = pytest.mark.gpu

R = 24
DX = 1.0 / R
DT = 1e-3
ORIGIN = (0.0, 0.0, 0.0)


def particles(n, seed, outside=()):
    rng = np.random.default_rng(seed)
    x = rng.uniform(3.5 * DX, (R - 4.5) * DX, (n, 3)).astype(np.float32)
    for i, pos in outside:
        x[i] = pos
    v = rng.standard_normal((n, 3)).astype(np.float32)
    C = (3.0 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    tau = (50.0 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    tau = 0.5 * (tau + tau.transpose(0, 2, 1))
    m = rng.uniform(0.5, 1.5, n).astype(np.float32) * 1e-3
    V0 = np.full(n, 1e-6, np.float32)
    F = (np.eye(3) + 0.05 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    return x, v, C, tau, m, V0, F


def device_transfer(x, v, C, tau, m, V0, F):
    import torch
    from baking_b200 import arrays
    from baking_b200.physics.grid import GridState, UpdateGrid
    from baking_b200.physics.transfer import GridToParticle, ParticleToGrid
    dev = torch.device("cuda:0")
    n = len(x)
    cfg = replace(SimulationConfig(), grid_resolution=R, grid_spacing=DX, time_step=DT, gravity=(0.0, -9.8, 0.0),
                  boundary_cells=3, device_name="cuda:0")
    grid = GridState(cfg, dev)
    flags = torch.zeros(2, dtype=torch.int32, device=dev)
    xd, vd = arrays.from_numpy(x, "f4", dev), arrays.from_numpy(v, "f4", dev)
    Cd, taud, Fd = arrays.from_numpy(C, "f4", dev), arrays.from_numpy(tau, "f4", dev), arrays.from_numpy(F, "f4", dev)
    md, V0d = arrays.from_numpy(m, "f4", dev), arrays.from_numpy(V0, "f4", dev)
    ParticleToGrid(xd, vd, Cd, taud, md, V0d, grid, ORIGIN, DX, R, DT, flags)
    node_pm = grid.node_pm.cpu().numpy().copy()
    UpdateGrid(grid, cfg)
    node_v = grid.node_v.cpu().numpy().copy()
    outs = [arrays.vec3s(n, device=dev, pitch=arrays.layout_pitch(xd) if n else None) for _ in range(2)]
    mats = [arrays.mat33s(n, device=dev, pitch=arrays.layout_pitch(xd) if n else None) for _ in range(2)]
    GridToParticle(xd, Fd, grid, outs[0], outs[1], mats[0], mats[1], ORIGIN, DX, R, DT, flags)
    torch.cuda.synchronize()
    return dict(node_pm=node_pm, node_v=node_v, x=arrays.to_numpy(outs[0]), v=arrays.to_numpy(outs[1]),
                C=arrays.to_numpy(mats[0]), F=arrays.to_numpy(mats[1]), flags=flags.cpu().numpy())


def oracle_transfer(x, v, C, tau, m, V0, F):
    n = len(x)
    nodes = R ** 3
    node_m, node_p, node_v = ora.f32(nodes), ora.f32(nodes, 3), ora.f32(nodes, 3)
    flags = ora.i32(2)
    origin = ora.vec(ORIGIN)
    gravity = ora.vec((0.0, -9.8, 0.0))
    L = ora.lib()
    L.ora_particle_to_grid(n, *(ora.ptr(np.ascontiguousarray(a), "f4") for a in (x, v, C, tau, m, V0)),
                           ora.ptr(node_m, "f4"), ora.ptr(node_p, "f4"), ora.ptr(origin, "f4"), DX, R, DT,
                           ora.ptr(flags, "i4"))
    L.ora_update_grid(nodes, ora.ptr(node_m, "f4"), ora.ptr(node_p, "f4"), ora.ptr(node_v, "f4"), R, 3,
                      ora.ptr(gravity, "f4"), DT)
    xo, vo, Co, Fo = ora.f32(n, 3), ora.f32(n, 3), ora.f32(n, 3, 3), ora.f32(n, 3, 3)
    L.ora_grid_to_particle(n, ora.ptr(np.ascontiguousarray(x), "f4"), ora.ptr(np.ascontiguousarray(F), "f4"),
                           ora.ptr(node_v, "f4"), ora.ptr(xo, "f4"), ora.ptr(vo, "f4"), ora.ptr(Co, "f4"),
                           ora.ptr(Fo, "f4"), ora.ptr(origin, "f4"), DX, R, DT, ora.ptr(flags, "i4"))
    return dict(node_m=node_m, node_p=node_p, node_v=node_v, x=xo, v=vo, C=Co, F=Fo, flags=flags)


def compare(dev, ora_out, valid):
    m_scale = max(float(np.abs(ora_out["node_m"]).max()), 1e-30)
    p_scale = max(float(np.abs(ora_out["node_p"]).max()), 1e-30)
    np.testing.assert_allclose(dev["node_pm"][:, 3], ora_out["node_m"], rtol=1e-5, atol=1e-6 * m_scale)
    np.testing.assert_allclose(dev["node_pm"][:, :3], ora_out["node_p"], rtol=1e-5, atol=1e-6 * p_scale)
    v_scale = max(float(np.abs(ora_out["node_v"]).max()), 1e-30)
    np.testing.assert_allclose(dev["node_v"][:, :3], ora_out["node_v"], rtol=1e-4, atol=1e-5 * v_scale)
    for key in ("x", "v", "C", "F"):
        a, b = dev[key][valid], ora_out[key][valid]
        scale = max(float(np.abs(b).max()), 1e-30) if b.size else 1.0
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-5 * scale, err_msg=key)


@pytest.mark.parametrize("n", [0, 1, 31, 33, 257, 1000])
def test_ragged_particle_counts(n):
    arrs = particles(n, seed=n + 3)
    dev, ref = device_transfer(*arrs), oracle_transfer(*arrs)
    compare(dev, ref, np.ones(n, dtype=bool))
    assert dev["flags"].tolist() == ref["flags"].tolist() == [0, 0]
    if n == 0:
        assert not dev["node_pm"].any()


def test_stencil_leaving_the_grid_is_flagged_and_skipped():
    n = 100
    outside = [(7, (0.2 * DX, 0.5, 0.5)), (42, (0.5, (R - 1.2) * DX, 0.5)), (99, (0.5, 0.5, -DX))]
    arrs = particles(n, seed=5, outside=outside)
    dev, ref = device_transfer(*arrs), oracle_transfer(*arrs)
    assert dev["flags"][1] == 1 and ref["flags"][1] == 1
    valid = np.ones(n, dtype=bool)
    valid[[i for i, _ in outside]] = False
    compare(dev, ref, valid)


def test_wall_clamp_in_boundary_cells():
    """Particles in the boundary layer moving into the walls: the outward node velocities are
    clamped to zero on both engines (grid.py:29-37)."""
    n = 64
    rng = np.random.default_rng(9)
    x, v, C, tau, m, V0, F = particles(n, seed=9)
    x[:32] = rng.uniform(1.6 * DX, 2.4 * DX, (32, 3)).astype(np.float32)   # near the low walls
    v[:32] = -5.0
    x[32:] = rng.uniform((R - 3.4) * DX, (R - 2.6) * DX, (32, 3)).astype(np.float32)  # near the high walls
    v[32:] = 5.0
    arrs = (x, v, C, tau, m, V0, F)
    dev, ref = device_transfer(*arrs), oracle_transfer(*arrs)
    compare(dev, ref, np.ones(n, dtype=bool))
    nv = dev["node_v"][:, :3].reshape(R, R, R, 3)
    assert (nv[:3, :, :, 0] >= 0).all() and (nv[R - 3:, :, :, 0] <= 0).all()
