"""Reverse-mode derivatives of substeps, behind ``torch.autograd``.

The reference differentiates a run by recording ``MpmSimulator.Step()`` calls on a Warp tape
(``retain_history=True`` keeps every state and grid alive, physics/mpm.py:170-178) and replaying
the generated kernel adjoints (tests/test_warp_autodiff.py:27-49, tests/test_ding.py:140-161,
tests/test_ding_thermal.py:160-190). Here :func:`Rollout` runs ``steps`` substeps of an
``MpmSimulator`` as one autograd node:

* forward: the fused substep kernels, keeping a copy of the primary state every
  ``checkpoint_every`` substeps (no per-step history);
* backward: per checkpoint segment, latest first, the segment's substeps are re-run from its
  checkpoint, each on a grid of its own so that the grid (with transport, also its node fields)
  stays for its reverse step; each substep is then reversed by ``bk_substep_adjoint`` (G2P +
  return map with, in gas mode, the coupled end-state porosity solve, grid update, P2G) and, with
  transport, by ``bk_transport_adjoint`` (scalar G2P with the water stress and particle mass, the
  gas source and gas-pressure stress, diffusion, scalar P2G, surface heat and loss through the
  mesh face areas).

Memory is one state per checkpoint plus ``checkpoint_every`` states and grids, instead of one
state and one grid per substep. Covered: neo-Hookean and Ding materials, with or without
thermal-water transport and gas, after settling. Gradients reach the initial positions,
velocities, affine velocities, deformation gradients, Ding elastic gradients, stresses and
porosities, the material temperatures without transport or the transport temperatures and water
masses with it, the gas content, the viscosity parameter, Young's modulus, the heat-transfer
parameter and the gas source rates (one shared or one per particle).
Discrete switches (gelation latch, wall clamping, stencil validity, tray contact, nodes without
capacity) carry no gradient, as in the reference.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import replace

import torch

from .. import _lib, arrays
from .materials.ding import DingMaterial
from .substep import PHASE_MECHANICS, PHASE_TRANSPORT, BkConstants, BkSurface, state_struct

P = C.c_void_p


class BkAdjointState(C.Structure):
    _fields_ = [("x", P), ("v", P), ("C", P), ("F", P), ("Fe", P), ("tau", P), ("porosity", P),
                ("temperature", P), ("mass", P)]


class BkAdjointTransport(C.Structure):
    _fields_ = [("temperature_out", P), ("water_out", P), ("temperature_in", P), ("water_in", P),
                ("node_dT_ratio", P), ("node_fields", P * 6), ("vertices", P), ("heat_parameter", P),
                ("gas_moles_out", P), ("gas_moles_in", P), ("gas_rate", P)]


_SIGNATURE = [P] * 11 + [P]
_SIGNATURES = {
    "bk_substep_adjoint": _SIGNATURE,
    "bk_transport_adjoint_prepare": [P] * 7 + [P],
    "bk_transport_adjoint": [P] * 7 + [P],
}

# (keyword, state attribute); outputs follow the same order.
_KINEMATIC = (("positions", "particle_positions"), ("velocities", "particle_velocities"),
              ("affine_velocities", "affine_velocities"), ("deformation_gradients", "deformation_gradients"))
_DING = (("elastic_gradients", "elastic_gradients"), ("kirchhoff_stresses", "kirchhoff_stresses"),
         ("porosities", "porosities"), ("temperatures", "temperatures"))
_DING_DISCRETE = ("gelled",)
_GAS = (("gas_moles", "gas_moles"),)
_TRANSPORT = (("transport_temperatures", "temperatures"), ("water_masses", "water_masses"))


def _declare(lib):
    for name, argtypes in _SIGNATURES.items():
        fn = getattr(lib, name)
        if fn.argtypes != argtypes:
            fn.restype = C.c_int
            fn.argtypes = argtypes
    return lib.bk_substep_adjoint


def _p(t):
    return None if t is None else t.data_ptr()


def _keys(is_ding, transport, gas=False):
    return [k for k, _ in _KINEMATIC] + ([k for k, _ in _DING] if is_ding else []) + \
        ([k for k, _ in _GAS] if gas else []) + ([k for k, _ in _TRANSPORT] if transport else [])


def _arrays_of(state, is_ding, transport, gas=False):
    """The primary arrays of a state: kinematic, Ding (then the gelation latch), gas, transport."""
    out = [getattr(state, attr) for _, attr in _KINEMATIC]
    if is_ding:
        m = state.material_state
        out += [getattr(m, attr) for _, attr in _DING] + [getattr(m, a) for a in _DING_DISCRETE]
        if gas:
            out += [getattr(m, attr) for _, attr in _GAS]
    if transport:
        t = state.transport_state
        out += [getattr(t, attr) for _, attr in _TRANSPORT]
    return out


def _outputs_of(state, is_ding, transport, gas=False):
    """The differentiable arrays of a state, in the order of ``_keys``."""
    arrs = _arrays_of(state, is_ding, transport, gas)
    return arrs[:8] + arrs[9:] if is_ding else arrs


def _copy_state(dst, src, is_ding, transport, gas=False):
    for d, s in zip(_arrays_of(dst, is_ding, transport, gas), _arrays_of(src, is_ding, transport, gas)):
        d.copy_(s)


class _AdjointBuffers:
    """Adjoint state in the plane layout (updated in place, substep by substep)."""

    def __init__(self, n, pitch, device, is_ding, transport, gas=False):
        self.x = arrays.vec3s(n, device=device, pitch=pitch)
        self.v = arrays.vec3s(n, device=device, pitch=pitch)
        self.C = arrays.mat33s(n, device=device, pitch=pitch)
        self.F = arrays.mat33s(n, device=device, pitch=pitch)
        self.Fe = arrays.mat33s(n, device=device, pitch=pitch) if is_ding else None
        self.tau = arrays.mat33s(n, device=device, pitch=pitch) if is_ding else None
        self.porosity = arrays.scalars(n, device=device, pitch=pitch) if is_ding else None
        self.temperature = arrays.scalars(n, device=device, pitch=pitch) if is_ding else None
        self.mass = arrays.scalars(n, device=device, pitch=pitch) if transport else None
        self.N = arrays.scalars(n, torch.float64, device) if gas else None
        self.T = arrays.scalars(n, torch.float64, device) if transport else None
        self.W = arrays.scalars(n, torch.float64, device) if transport else None

    def tensors(self):
        """In the order of ``_keys``."""
        out = [self.x, self.v, self.C, self.F]
        if self.Fe is not None:
            out += [self.Fe, self.tau, self.porosity, self.temperature]
        if self.N is not None:
            out.append(self.N)
        if self.T is not None:
            out += [self.T, self.W]
        return out

    def struct(self):
        s = BkAdjointState()
        s.x, s.v, s.C, s.F = _p(self.x), _p(self.v), _p(self.C), _p(self.F)
        s.Fe, s.tau, s.porosity, s.temperature = _p(self.Fe), _p(self.tau), _p(self.porosity), _p(self.temperature)
        s.mass = _p(self.mass)
        return s


class _Runner:
    """Forward run with checkpoints and the reverse sweep for one ``Rollout`` call."""

    def __init__(self, sim, steps, checkpoint_every):
        self.is_ding = isinstance(sim.material, DingMaterial)
        self.transport = sim.transport is not None
        self.gas = bool(self.is_ding and sim.material.ding_config.gas_enabled)
        if self.transport and not self.is_ding:
            raise NotImplementedError("with transport the adjoint needs the ding2019 material")
        if sim.IsSettling:
            raise NotImplementedError("Rollout starts after settling (settling substeps have no adjoint here)")
        if steps < 1 or checkpoint_every < 1:
            raise ValueError("steps and checkpoint_every must be positive")
        self.sim = sim
        self.steps = int(steps)
        self.every = int(checkpoint_every)
        self.engine = sim._engine
        self.lib = _lib.load()
        self.fn = _declare(self.lib)
        self.checkpoints = []

    # ------------------------------------------------------------- buffers
    def _pool(self):
        """Buffers kept on the simulator between Rollout calls (states, grids, adjoint arrays)."""
        return self.sim._buffers.setdefault("rollout", {"snapshots": [], "work": [], "grids": []})

    def _states(self, key, count):
        lst = self._pool()[key]
        while len(lst) < count:
            lst.append(self.sim._allocate_like_current(share_accumulators=False))
        return lst

    # ----------------------------------------------------------------- forward
    def _snapshot(self, state):
        snaps = self._states("snapshots", len(self.checkpoints) + 1)
        snap = snaps[len(self.checkpoints)]
        _copy_state(snap, state, self.is_ding, self.transport, self.gas)
        return snap

    def _set_young_modulus(self, E):
        mat = self.sim.material
        mat.material_config = replace(mat.material_config, young_modulus=float(E))

    def forward(self, inputs):
        sim = self.sim
        if self.transport and inputs.get("temperatures") is not None:
            raise ValueError("with transport set transport_temperatures (the material temperature follows them)")
        state = sim.current_state
        for name, target in zip(_keys(self.is_ding, self.transport, self.gas),
                                _outputs_of(state, self.is_ding, self.transport, self.gas)):
            value = inputs.get(name)
            if value is not None:
                target.copy_(value.detach().reshape(target.shape))
        if inputs.get("viscosity_parameter") is not None:
            if not self.is_ding:
                raise ValueError("viscosity_parameter needs the ding2019 material")
            sim.material.viscosity_parameter.copy_(inputs["viscosity_parameter"].detach().reshape(1))
        if inputs.get("gas_source_rates") is not None:
            if not self.gas:
                raise ValueError("gas_source_rates needs gas mode")
            sim.SetGasSourceRates(inputs["gas_source_rates"].detach().reshape(-1).cpu().numpy())
        if inputs.get("heat_transfer_parameter") is not None:
            if not self.transport:
                raise ValueError("heat_transfer_parameter needs transport")
            sim.transport.heat_transfer_parameter.copy_(inputs["heat_transfer_parameter"].detach().reshape(1))
        if inputs.get("young_modulus") is not None:
            self._set_young_modulus(inputs["young_modulus"].detach().reshape(()).item())
        self.checkpoints = [self._snapshot(state)]
        for k in range(self.steps):
            sim._substep(check=False)
            if (k + 1) % self.every == 0 and k + 1 < self.steps:
                self.checkpoints.append(self._snapshot(sim._current))
        messages = sim._device_flag_messages()
        flags = sim.error_flags.tolist()
        if flags[0]:
            messages.insert(0, "nonpositive/nonfinite J; reduce dt or inspect loading and sampling")
        if flags[1]:
            messages.insert(0, "particle stencil left the grid; enlarge the domain or reduce dt")
        if messages:
            raise RuntimeError(messages[0] + " (during Rollout)")
        final = sim.current_state  # with transport this also fills the material temperature from T
        return tuple(t.detach().clone() for t in _outputs_of(final, self.is_ding, self.transport, self.gas))

    # ---------------------------------------------------------------- backward
    def _check(self, rc, name):
        if rc != 0:
            raise RuntimeError(f"{name} failed ({rc}): {self.lib.bk_last_error().decode(errors='replace')}")

    def _transport_buffers(self, pool):
        """Node and vertex adjoint scratch (zero between calls) and a private surface whose vertex
        and owner heat/loss buffers the recomputed substeps write instead of the simulator's."""
        if pool.get("transport") is not None:
            return pool["transport"]
        eng, dev = self.engine, self.sim.device
        n, pitch, R = eng.n, eng.pitch, self.sim.simulation_config.grid_resolution
        t = dict(node_dT=torch.zeros(R ** 3, 2, dtype=torch.float64, device=dev),
                 node_fields=[torch.zeros(R ** 3, dtype=torch.float64, device=dev) for _ in range(6)],
                 vertices=torch.zeros(3, max(int(eng.surface.vertex_pitch), 1), dtype=torch.float64, device=dev),
                 T_mat=arrays.scalars(n, device=dev, pitch=pitch),
                 mass=arrays.scalars(n, device=dev, pitch=pitch),
                 tau=arrays.mat33s(n, device=dev, pitch=pitch))
        surface = BkSurface.from_buffer_copy(eng.surface)
        if eng.surface.owner_count > 0:
            src = eng._surface_tensors
            t["owner_heat"] = torch.zeros_like(src["owner_heat"])
            t["owner_loss"] = torch.zeros_like(src["owner_loss"])
            surface.owner_heat, surface.owner_loss = _p(t["owner_heat"]), _p(t["owner_loss"])
        if eng.surface.vertex_count > 0:
            # Plane layout with the surface's vertex pitch, as the vertex kernels index it
            # (empty_like of the strided view would return a row-major n x 3 buffer).
            verts = self.sim.surface_vertices_buffer()
            t["surface_vertices"] = arrays.vec3s(verts.shape[0], device=dev, pitch=int(eng.surface.vertex_pitch))
            surface.vertices = _p(t["surface_vertices"])
        t["surface"] = surface
        pool["transport"] = t
        return t

    def backward(self, grads):
        pool = self._pool()
        try:
            return self._backward(grads, pool)
        except Exception:
            # A sweep cut short leaves grid fields and node scratch nonzero: start over next time.
            for key in ("grids", "adjoint", "transport"):
                pool.pop(key, None)
            pool["grids"] = []
            raise

    def _backward(self, grads, pool):
        sim, eng = self.sim, self.engine
        n, pitch, dev = eng.n, eng.pitch, sim.device
        R = sim.simulation_config.grid_resolution
        if pool.get("adjoint") is None:
            pool["adjoint"] = _AdjointBuffers(n, pitch, dev, self.is_ding, self.transport, self.gas)
            # node_v_adj must be zero before the first call; each call leaves it zero (node box mode).
            pool["node_v_adj"] = torch.zeros(R ** 3, 4, dtype=torch.float32, device=dev)
            pool["node_pm_adj"] = torch.empty(R ** 3, 4, dtype=torch.float32, device=dev)
        adj, node_v_adj, node_pm_adj = pool["adjoint"], pool["node_v_adj"], pool["node_pm_adj"]
        for buf, g in zip(adj.tensors(), grads):
            if g is None:
                buf.zero_()
            else:
                buf.copy_(g.reshape(buf.shape))
        if self.transport:
            # The final material temperature is float(T'): its gradient joins that of T'.
            adj.T += adj.temperature.double()
            adj.temperature.zero_()
        params_adj = torch.zeros(4, dtype=torch.float64, device=dev)  # mu, lambda, eta, heat parameter
        rate_adj = None
        if self.gas:
            rate_adj = torch.zeros(sim.material.production_parameter.shape[0], dtype=torch.float64, device=dev)
        p = eng.params(False)
        cst = eng.constants(False)
        stream = _lib.stream_handle()
        span = min(self.every, self.steps)
        # One grid per substep of a segment: the forward run of substep t leaves its grid (and, in
        # bounds[6:12], its active box; with transport, its node fields) for the reverse of substep t.
        grids = pool["grids"]
        while len(grids) < span:
            grids.append(eng.mechanics_grid(own_transport=self.transport))
        work = self._states("work", span + 1)
        adj_struct = adj.struct()
        phases = PHASE_MECHANICS
        surface = eng.surface
        if self.transport:
            phases |= PHASE_TRANSPORT
            tb = self._transport_buffers(pool)
            surface = tb["surface"]
            tadj = BkAdjointTransport()
            tadj.temperature_out = tadj.temperature_in = _p(adj.T)
            tadj.water_out = tadj.water_in = _p(adj.W)
            tadj.node_dT_ratio = _p(tb["node_dT"])
            for k in range(6):
                tadj.node_fields[k] = _p(tb["node_fields"][k])
            tadj.vertices = _p(tb["vertices"])
            tadj.heat_parameter = params_adj.data_ptr() + 3 * 8
            if self.gas:
                tadj.gas_moles_out = tadj.gas_moles_in = _p(adj.N)
                tadj.gas_rate = _p(rate_adj)
            # P2G of a transport substep uses T', dry + W' and the water-stressed stress.
            cst_mech = BkConstants.from_buffer_copy(cst)
            cst_mech.mass = _p(tb["mass"])
        for seg in range(len(self.checkpoints) - 1, -1, -1):
            first = seg * self.every
            length = min(self.every, self.steps - first)
            _copy_state(work[0], self.checkpoints[seg], self.is_ding, self.transport, self.gas)
            for t in range(length):
                self._run(work[t], work[t + 1], phases, grids[t][0], surface)
            for t in range(length - 1, -1, -1):
                grid, g = grids[t]
                sin = state_struct(work[t], self.is_ding, self.transport, self.gas)
                if self.transport:
                    self._check(self.lib.bk_transport_adjoint_prepare(
                        C.byref(p), C.byref(sin), C.byref(cst), _p(g["node_dT_ratio"]), _p(tb["T_mat"]),
                        _p(tb["mass"]), _p(tb["tau"]), stream), "bk_transport_adjoint_prepare")
                    smech = state_struct(work[t], self.is_ding, self.transport, self.gas)
                    smech.tau, smech.material_temperature = _p(tb["tau"]), _p(tb["T_mat"])
                    self._check(self.fn(C.byref(p), C.byref(smech), C.byref(cst_mech), _p(g["node_pm"]),
                                        _p(g["node_v"]), g["bounds"].data_ptr() + 6 * 4, C.byref(adj_struct),
                                        C.byref(adj_struct), _p(node_v_adj), _p(node_pm_adj), _p(params_adj),
                                        stream), "bk_substep_adjoint")
                    self._check(self.lib.bk_transport_adjoint(
                        C.byref(p), C.byref(sin), C.byref(cst), C.byref(grid), C.byref(surface),
                        C.byref(adj_struct), C.byref(tadj), stream), "bk_transport_adjoint")
                else:
                    self._check(self.fn(C.byref(p), C.byref(sin), C.byref(cst), _p(g["node_pm"]), _p(g["node_v"]),
                                        g["bounds"].data_ptr() + 6 * 4, C.byref(adj_struct), C.byref(adj_struct),
                                        _p(node_v_adj), _p(node_pm_adj), _p(params_adj), stream),
                                "bk_substep_adjoint")
        self.checkpoints = []
        return adj, params_adj, rate_adj

    def _run(self, state_in, state_out, phases, grid, surface):
        eng = self.engine
        if not self.transport:
            eng.run(state_in, state_out, False, phases, False, grid=grid)
            return
        saved = eng.surface
        eng.surface = surface
        try:
            eng.run(state_in, state_out, False, phases, False, grid=grid, keep_fields=True)
        finally:
            eng.surface = saved


class _RolloutFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, runner, names, *values):
        ctx.runner = runner
        ctx.names = names
        ctx.shapes = [None if v is None else v.shape for v in values]
        return runner.forward(dict(zip(names, values)))

    @staticmethod
    def backward(ctx, *grads):
        runner = ctx.runner
        adj, params_adj, rate_adj = runner.backward(grads)
        state_grads = dict(zip(_keys(runner.is_ding, runner.transport, runner.gas), adj.tensors()))
        nu = runner.sim.material.material_config.poisson_ratio
        mu_bar, lam_bar, eta_bar, h_bar = params_adj.tolist()
        dev = runner.sim.device
        out = []
        for name, shape in zip(ctx.names, ctx.shapes):
            if shape is None:
                out.append(None)
            elif name in state_grads:
                out.append(state_grads[name].clone().reshape(shape))
            elif name == "viscosity_parameter":
                out.append(torch.full(shape, eta_bar, dtype=torch.float32, device=dev))
            elif name == "gas_source_rates":
                out.append(rate_adj.float().reshape(shape).clone())
            elif name == "heat_transfer_parameter":
                out.append(torch.full(shape, h_bar, dtype=torch.float32, device=dev))
            elif name == "young_modulus":
                e_bar = mu_bar / (2.0 * (1.0 + nu)) + lam_bar * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
                out.append(torch.full(shape, e_bar, dtype=torch.float32, device=dev))
            else:
                out.append(None)
        return (None, None, *out)


_INPUTS = tuple(k for k, _ in _KINEMATIC) + tuple(k for k, _ in _DING) + tuple(k for k, _ in _GAS) + \
    tuple(k for k, _ in _TRANSPORT) + ("viscosity_parameter", "young_modulus", "heat_transfer_parameter",
                                      "gas_source_rates")


def Rollout(sim, steps, checkpoint_every=16, **inputs):
    """Run ``steps`` substeps of ``sim`` as one differentiable torch operation.

    Keyword inputs (any subset; each may require grad) replace the corresponding values before the
    first substep: ``positions``, ``velocities`` (n, 3); ``affine_velocities``,
    ``deformation_gradients`` (n, 3, 3); for the Ding model ``elastic_gradients``,
    ``kirchhoff_stresses`` (n, 3, 3), ``porosities`` (n,), ``temperatures`` (n,; the material
    temperature, without transport only) and ``viscosity_parameter`` (1,); with transport
    ``transport_temperatures``, ``water_masses`` (n,, float64) and ``heat_transfer_parameter`` (1,);
    in gas mode ``gas_moles`` (n,, float64) and ``gas_source_rates`` ((1,) or (n,), as
    ``SetGasSourceRates``); ``young_modulus`` (scalar or (1,)). Returns a dict of the final state's
    arrays (detached copies joined to the autograd graph): the four kinematic arrays; for Ding
    ``elastic_gradients``, ``kirchhoff_stresses``, ``porosities``, ``temperatures``; in gas mode
    ``gas_moles``; with transport ``transport_temperatures`` and ``water_masses``. The simulator advances by ``steps`` substeps
    as ``AdvanceUnchecked`` would, and its parameters keep the values given. Device flags raised
    during the run raise ``RuntimeError``.
    """
    unknown = set(inputs) - set(_INPUTS)
    if unknown:
        raise TypeError(f"unknown Rollout inputs: {sorted(unknown)}")
    runner = _Runner(sim, steps, checkpoint_every)
    names = tuple(k for k in _INPUTS if k in inputs)
    values = tuple(inputs[k] for k in names)
    outputs = _RolloutFunction.apply(runner, names, *values)
    return dict(zip(_keys(runner.is_ding, runner.transport, runner.gas), outputs))
