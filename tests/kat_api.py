"""One interface over the two engines the known-answer tests run on.

``oracle``: the CPU restatement (``oracle/``), the checker. ``cuda``: the product
(``baking_b200``) on a B200. The known answers come from the reference's own tests;
each test module cites the reference test it restates.
"""
from dataclasses import replace

import numpy as np
import pytest

from tests.scenes import assign, to_np

GPU_PARAM = pytest.param("cuda", marks=pytest.mark.gpu)
ENGINES = ["oracle", GPU_PARAM]


class Api:
    def __init__(self, engine):
        self.engine = engine
        if engine == "oracle":
            from oracle import sim as osim
            self.m = osim
            self.Simulator = osim.OracleSimulator
            self.device = "cpu"
        else:
            from baking_b200.physics import mpm, state
            from baking_b200.physics.materials import ding
            self.mpm, self.state_mod, self.ding = mpm, state, ding
            self.Simulator = mpm.MpmSimulator
            self.device = "cuda:0"

    # -- configuration
    def sim_config(self, **kwargs):
        from baking_b200.config import SimulationConfig
        return replace(SimulationConfig(), device_name=self.device, **kwargs)

    def simulator(self, mesh, samples, sim_config, material_config, *args, **kwargs):
        return self.Simulator(mesh, samples, sim_config, material_config, *args, **kwargs)

    # -- point material tests
    def ding_material(self, material_config, ding_config, initial_temperature_k=293.15):
        if self.engine == "oracle":
            return self.m.DingMaterial(material_config, ding_config, False, initial_temperature_k)
        return self.ding.DingMaterial(material_config, ding_config, self.device, False, initial_temperature_k)

    def allocate(self, n):
        if self.engine == "oracle":
            return self.m.AllocateState(n)
        return self.state_mod.AllocateState(n, self.device)

    def point(self, material):
        state = self.allocate(1)
        assign(state.deformation_gradients, np.eye(3, dtype=np.float32)[None])
        material.InitializeState(state)
        return state

    def point_step(self, material, old, total_gradient, time_step=0.01, check=True):
        out = self.allocate(1)
        increment = total_gradient @ np.linalg.inv(to_np(old.deformation_gradients)[0])
        assign(out.deformation_gradients, total_gradient.astype(np.float32)[None])
        assign(out.affine_velocities, ((increment - np.eye(3)) / time_step).astype(np.float32)[None])
        material.AdvanceState(old, out, time_step)
        if check:
            material.CheckState()
        return out

    # -- kernels used directly by the reference tests
    def diffuse_grid(self, vol, cap, T, s, water, heat, loss, exch, dT, dW, errors, *scalars):
        if self.engine == "oracle":
            from oracle import ora
            ora.diffuse_grid(vol, cap, T, s, water, heat, loss, exch, dT, dW, errors, *scalars)
        else:
            from baking_b200.physics.thermal_water import DiffuseGrid
            DiffuseGrid(vol, cap, T, s, water, heat, loss, exch, dT, dW, errors, *scalars)

    def array(self, values, kind):
        if self.engine == "oracle":
            dtype = {"f4": np.float32, "f8": np.float64, "i4": np.int32}[kind]
            return np.array(values, dtype=dtype, order="C", copy=True)
        from baking_b200 import arrays
        return arrays.from_numpy(np.asarray(values), kind, self.device)

    def zeros(self, shape, kind):
        dtype = {"f4": np.float32, "f8": np.float64, "i4": np.int32}[kind]
        return self.array(np.zeros(shape, dtype=dtype), kind)
