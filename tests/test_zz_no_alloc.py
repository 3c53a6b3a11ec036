"""bk_substep_static_grid -- the mechanics substep for callers that cannot allocate device memory.

It must give the same particle state as bk_substep with a caller-allocated grid, for two
substeps in a row (the second call finds the shared static grid holding the first call's nodes,
so it also checks that each call resets what it uses), on the demo grid (40^3) and on the largest
grid the array holds (48^3, where the velocity nodes and the box bounds sit at the array's end).
The second call must leave the device's free memory unchanged: that is the property the entry
point exists for. Both entry points are called directly
through the C ABI on the same inputs. Float atomics accumulate in a different order in the two
runs, so results agree to the parity tolerance used elsewhere (1e-5 relative), not bit for bit.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _scene(resolution=40):
    from dataclasses import replace
    from baking_b200.config import DingConfig, MaterialConfig, SimulationConfig
    from baking_b200.geometry import CreateDemoMesh, SampleParticles
    from baking_b200.physics.mpm import MpmSimulator
    mesh = CreateDemoMesh(3)
    cfg = replace(SimulationConfig(), device_name="cuda:0", grid_resolution=resolution, grid_spacing=1.0 / resolution)
    sim = MpmSimulator(mesh, SampleParticles(mesh, 1000.0, 4), cfg,
                       MaterialConfig(model="ding2019"), initial_velocity=(0.3, -0.2, 0.1),
                       ding_config=DingConfig(yield_stress=300.0, viscosity=1e6))
    rng = np.random.default_rng(5)
    rates = (rng.standard_normal((3, 3)) * 2.0).astype(np.float32)
    st = sim.current_state
    st.affine_velocities.copy_(torch.as_tensor(np.tile(rates, (st.affine_velocities.shape[0], 1, 1)),
                                               device=st.affine_velocities.device))
    return sim


def _grid(R, device):
    empty = [2 ** 31 - 1] * 3 + [-2 ** 31] * 3
    return (torch.zeros(R ** 3, 4, device=device), torch.zeros(R ** 3, 4, device=device),
            torch.tensor(empty + empty, dtype=torch.int32, device=device))


@pytest.mark.parametrize("resolution", [40, 48])
def test_static_grid_substep_matches_allocated_grid_twice(resolution):
    from baking_b200 import _lib
    from baking_b200.physics import substep as sub
    sim = _scene(resolution)
    lib = _lib.load()
    fn = lib.bk_substep_static_grid
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 7
    eng = sim._engine
    params, consts = eng.params(False), eng.constants(False)
    dev = sim.device
    start = sim.current_state
    results = {}
    for path in ("allocated", "static"):
        state_in = start
        outs = []
        for call in range(2):
            out = sim._allocate_like_current()
            flags = sub.BkFlags()
            flag_arrays = [torch.zeros(k, dtype=torch.int32, device=dev) for k in (2, 3, 2)]
            flags.simulation, flags.ding, flags.transport = [t.data_ptr() for t in flag_arrays]
            diag = sub.BkDiagnostics()
            residuals = torch.zeros(2, device=dev)
            diag.max_residuals = residuals.data_ptr()
            s_in = sub.state_struct(state_in, True, False, False)
            s_out = sub.state_struct(out, True, False, False)
            stream = _lib.stream_handle()
            if path == "allocated":
                pm, v, bounds = _grid(sim.simulation_config.grid_resolution, dev)
                grid = sub.BkGrid()
                grid.node_pm, grid.node_v, grid.bounds = pm.data_ptr(), v.data_ptr(), bounds.data_ptr()
                rc = lib.bk_substep(C.byref(params), C.byref(s_in), C.byref(s_out), C.byref(consts), C.byref(grid),
                                    None, C.byref(diag), C.byref(flags), sub.PHASE_MECHANICS, stream)
            else:
                torch.cuda.synchronize()
                free_before = torch.cuda.mem_get_info()[0]
                rc = fn(C.byref(params), C.byref(s_in), C.byref(s_out), C.byref(consts), C.byref(diag), C.byref(flags),
                        stream)
                torch.cuda.synchronize()
                if call == 1:
                    assert torch.cuda.mem_get_info()[0] == free_before, "the second call changed free device memory"
            assert rc == 0, lib.bk_last_error().decode()
            torch.cuda.synchronize()
            assert all(int(t.sum()) == 0 for t in flag_arrays)
            outs.append(out)
            state_in = out
        results[path] = outs
    for call in range(2):
        a, b = results["allocated"][call], results["static"][call]
        for name in ("particle_positions", "particle_velocities", "affine_velocities", "deformation_gradients"):
            x, y = getattr(a, name).cpu().numpy(), getattr(b, name).cpu().numpy()
            np.testing.assert_allclose(y, x, rtol=1e-5, atol=1e-5 * np.abs(x).max(), err_msg=f"{name}, call {call}")
        for name in ("elastic_gradients", "porosities"):
            x = getattr(a.material_state, name).cpu().numpy()
            y = getattr(b.material_state, name).cpu().numpy()
            np.testing.assert_allclose(y, x, rtol=1e-5, atol=1e-5 * max(np.abs(x).max(), 1e-30),
                                       err_msg=f"{name}, call {call}")
        # Kirchhoff stress is (2 mu + 3 lambda)-scaled log strain of float32 singular values near 1,
        # resolved only to ~1e-7 strain; a stress floor of one microstrain covers that resolution.
        mc = sim.material.material_config
        floor = (2 * mc.shear_modulus + 3 * mc.lame_lambda) * 1e-6
        x, y = a.material_state.kirchhoff_stresses.cpu().numpy(), b.material_state.kirchhoff_stresses.cpu().numpy()
        np.testing.assert_allclose(y, x, rtol=1e-5, atol=floor, err_msg=f"kirchhoff_stresses, call {call}")


def test_static_grid_rejects_oversized_grid():
    from baking_b200 import _lib
    from baking_b200.physics import substep as sub
    sim = _scene()
    lib = _lib.load()
    fn = lib.bk_substep_static_grid
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 7
    params = sim._engine.params(False)
    params.resolution = 49
    rc = fn(C.byref(params), C.byref(sub.BkState()), C.byref(sub.BkState()), C.byref(sub.BkConstants()),
            C.byref(sub.BkDiagnostics()), C.byref(sub.BkFlags()), None)
    assert rc != 0
    assert "resolution 49" in lib.bk_last_error().decode()


@pytest.mark.parametrize("mode", ["transport", "gas"])
def test_static_grid_rejects_transport_and_gas(mode):
    from baking_b200 import _lib
    from baking_b200.physics import substep as sub
    sim = _scene()
    lib = _lib.load()
    fn = lib.bk_substep_static_grid
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 7
    params = sim._engine.params(False)
    setattr(params, mode, 1)
    rc = fn(C.byref(params), C.byref(sub.BkState()), C.byref(sub.BkState()), C.byref(sub.BkConstants()),
            C.byref(sub.BkDiagnostics()), C.byref(sub.BkFlags()), None)
    assert rc != 0
    assert "mechanics nodes only" in lib.bk_last_error().decode()
