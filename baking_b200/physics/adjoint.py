"""Reverse-mode derivatives of mechanics substeps, behind ``torch.autograd``.

The reference differentiates a run by recording ``MpmSimulator.Step()`` calls on a Warp tape
(``retain_history=True`` keeps every state and grid alive, physics/mpm.py:170-178) and replaying
the generated kernel adjoints (tests/test_warp_autodiff.py:27-49, tests/test_ding.py:140-161).
Here :func:`Rollout` runs ``steps`` substeps of an ``MpmSimulator`` as one autograd node:

* forward: the fused substep kernels, keeping a copy of the primary state every
  ``checkpoint_every`` substeps (no per-step history);
* backward: per checkpoint segment, latest first, the segment's states are recomputed from its
  checkpoint, and each substep is reversed by ``bk_substep_adjoint`` (hand-written adjoint
  kernels for G2P + return map, grid update and P2G) after re-running that substep's P2G and grid
  update to restore its grid.

Memory is one state per checkpoint plus ``checkpoint_every`` states, instead of one state and
one grid per substep. Covered: neo-Hookean and Ding (uncoupled porosity) materials without
transport or gas; gradients reach the initial positions, velocities, affine velocities,
deformation gradients, Ding elastic gradients, stresses, porosities and temperatures, the
viscosity parameter and Young's modulus. Discrete switches (gelation latch, wall clamping,
stencil validity) carry no gradient, as in the reference.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import replace

import torch

from .. import _lib, arrays
from .materials.ding import DingMaterial
from .substep import PHASE_MECHANICS, state_struct

P = C.c_void_p


class BkAdjointState(C.Structure):
    _fields_ = [("x", P), ("v", P), ("C", P), ("F", P), ("Fe", P), ("tau", P), ("porosity", P),
                ("temperature", P)]


_SIGNATURE = [P] * 11 + [P]

# (keyword, state attribute, material-state attribute); outputs follow the same order.
_KINEMATIC = (("positions", "particle_positions"), ("velocities", "particle_velocities"),
              ("affine_velocities", "affine_velocities"), ("deformation_gradients", "deformation_gradients"))
_DING = (("elastic_gradients", "elastic_gradients"), ("kirchhoff_stresses", "kirchhoff_stresses"),
         ("porosities", "porosities"), ("temperatures", "temperatures"))
_DING_DISCRETE = ("gelled",)


def _declare(lib):
    fn = lib.bk_substep_adjoint
    if fn.argtypes != _SIGNATURE:
        fn.restype = C.c_int
        fn.argtypes = _SIGNATURE
    return fn


def _p(t):
    return None if t is None else t.data_ptr()


def _arrays_of(state, is_ding):
    out = [getattr(state, attr) for _, attr in _KINEMATIC]
    if is_ding:
        m = state.material_state
        out += [getattr(m, attr) for _, attr in _DING] + [getattr(m, a) for a in _DING_DISCRETE]
    return out


def _copy_state(dst, src, is_ding):
    for d, s in zip(_arrays_of(dst, is_ding), _arrays_of(src, is_ding)):
        d.copy_(s)


class _AdjointBuffers:
    """Adjoint state in the plane layout (updated in place, substep by substep)."""

    def __init__(self, n, pitch, device, is_ding):
        self.x = arrays.vec3s(n, device=device, pitch=pitch)
        self.v = arrays.vec3s(n, device=device, pitch=pitch)
        self.C = arrays.mat33s(n, device=device, pitch=pitch)
        self.F = arrays.mat33s(n, device=device, pitch=pitch)
        self.Fe = arrays.mat33s(n, device=device, pitch=pitch) if is_ding else None
        self.tau = arrays.mat33s(n, device=device, pitch=pitch) if is_ding else None
        self.porosity = arrays.scalars(n, device=device, pitch=pitch) if is_ding else None
        self.temperature = arrays.scalars(n, device=device, pitch=pitch) if is_ding else None

    def tensors(self):
        out = [self.x, self.v, self.C, self.F]
        if self.Fe is not None:
            out += [self.Fe, self.tau, self.porosity, self.temperature]
        return out

    def struct(self):
        s = BkAdjointState()
        s.x, s.v, s.C, s.F = _p(self.x), _p(self.v), _p(self.C), _p(self.F)
        s.Fe, s.tau, s.porosity, s.temperature = _p(self.Fe), _p(self.tau), _p(self.porosity), _p(self.temperature)
        return s


class _Runner:
    """Forward run with checkpoints and the reverse sweep for one ``Rollout`` call."""

    def __init__(self, sim, steps, checkpoint_every):
        if sim.transport is not None:
            raise NotImplementedError("Rollout covers mechanics substeps; transport/gas runs have no adjoint here")
        if steps < 1 or checkpoint_every < 1:
            raise ValueError("steps and checkpoint_every must be positive")
        self.sim = sim
        self.steps = int(steps)
        self.every = int(checkpoint_every)
        self.is_ding = isinstance(sim.material, DingMaterial)
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
            lst.append(self.sim._allocate_like_current())
        return lst

    # ----------------------------------------------------------------- forward
    def _snapshot(self, state):
        snaps = self._states("snapshots", len(self.checkpoints) + 1)
        snap = snaps[len(self.checkpoints)]
        _copy_state(snap, state, self.is_ding)
        return snap

    def _set_young_modulus(self, E):
        mat = self.sim.material
        mat.material_config = replace(mat.material_config, young_modulus=float(E))

    def forward(self, inputs):
        sim = self.sim
        state = sim.current_state
        names = [k for k, _ in _KINEMATIC] + ([k for k, _ in _DING] if self.is_ding else [])
        targets = _arrays_of(state, self.is_ding)
        for name, target in zip(names, targets):
            value = inputs.get(name)
            if value is not None:
                target.copy_(value.detach().reshape(target.shape))
        if inputs.get("viscosity_parameter") is not None:
            if not self.is_ding:
                raise ValueError("viscosity_parameter needs the ding2019 material")
            sim.material.viscosity_parameter.copy_(inputs["viscosity_parameter"].detach().reshape(1))
        if inputs.get("young_modulus") is not None:
            self._set_young_modulus(inputs["young_modulus"].detach().reshape(()).item())
        if self.is_ding and sim.material.ding_config.gas_enabled:
            raise NotImplementedError("the gas (coupled porosity) return map has no adjoint here")
        self.checkpoints = []
        self.checkpoints.append(self._snapshot(state))
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
        final = sim.current_state
        return tuple(t.detach().clone() for t in _arrays_of(final, self.is_ding)[:8 if self.is_ding else 4])

    # ---------------------------------------------------------------- backward
    def backward(self, grads):
        sim, eng = self.sim, self.engine
        n, pitch, dev = eng.n, eng.pitch, sim.device
        pool = self._pool()
        if pool.get("adjoint") is None:
            R = sim.simulation_config.grid_resolution
            pool["adjoint"] = _AdjointBuffers(n, pitch, dev, self.is_ding)
            # node_v_adj must be zero before the first call; each call leaves it zero (node box mode).
            pool["node_v_adj"] = torch.zeros(R ** 3, 4, dtype=torch.float32, device=dev)
            pool["node_pm_adj"] = torch.empty(R ** 3, 4, dtype=torch.float32, device=dev)
        adj, node_v_adj, node_pm_adj = pool["adjoint"], pool["node_v_adj"], pool["node_pm_adj"]
        for buf, g in zip(adj.tensors(), grads):
            if g is None:
                buf.zero_()
            else:
                buf.copy_(g.reshape(buf.shape))
        params_adj = torch.zeros(3, dtype=torch.float64, device=dev)
        p = eng.params(False)
        cst = eng.constants(False)
        stream = _lib.stream_handle()
        span = min(self.every, self.steps)
        # One grid per substep of a segment: the forward run of substep t leaves its grid (and, in
        # bounds[6:12], its active box) for the adjoint of substep t.
        grids = pool["grids"]
        while len(grids) < span:
            grids.append(eng.mechanics_grid())
        work = self._states("work", span + 1)
        adj_struct = adj.struct()
        for seg in range(len(self.checkpoints) - 1, -1, -1):
            first = seg * self.every
            length = min(self.every, self.steps - first)
            _copy_state(work[0], self.checkpoints[seg], self.is_ding)
            for t in range(length):
                eng.run(work[t], work[t + 1], False, PHASE_MECHANICS, False, grid=grids[t][0])
            for t in range(length - 1, -1, -1):
                g = grids[t][1]
                sin = state_struct(work[t], self.is_ding, False, False)
                rc = self.fn(C.byref(p), C.byref(sin), C.byref(cst), _p(g["node_pm"]), _p(g["node_v"]),
                             g["bounds"].data_ptr() + 6 * 4, C.byref(adj_struct), C.byref(adj_struct),
                             _p(node_v_adj), _p(node_pm_adj), _p(params_adj), stream)
                if rc != 0:
                    raise RuntimeError(f"bk_substep_adjoint failed ({rc}): "
                                       f"{self.lib.bk_last_error().decode(errors='replace')}")
        self.checkpoints = []
        return adj, params_adj


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
        adj, params_adj = runner.backward(grads)
        state_grads = dict(zip([k for k, _ in _KINEMATIC] + [k for k, _ in _DING], adj.tensors()))
        mc = runner.sim.material.material_config
        nu = mc.poisson_ratio
        mu_bar, lam_bar, eta_bar = params_adj.tolist()
        out = []
        for name, shape in zip(ctx.names, ctx.shapes):
            if shape is None:
                out.append(None)
            elif name in state_grads:
                out.append(state_grads[name].clone().reshape(shape))
            elif name == "viscosity_parameter":
                out.append(torch.full(shape, eta_bar, dtype=torch.float32, device=runner.sim.device))
            elif name == "young_modulus":
                e_bar = mu_bar / (2.0 * (1.0 + nu)) + lam_bar * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
                out.append(torch.full(shape, e_bar, dtype=torch.float32, device=runner.sim.device))
            else:
                out.append(None)
        return (None, None, *out)


_INPUTS = tuple(k for k, _ in _KINEMATIC) + tuple(k for k, _ in _DING) + ("viscosity_parameter", "young_modulus")


def Rollout(sim, steps, checkpoint_every=16, **inputs):
    """Run ``steps`` substeps of ``sim`` as one differentiable torch operation.

    Keyword inputs (any subset; each may require grad) replace the corresponding values before the
    first substep: ``positions``, ``velocities`` (n, 3); ``affine_velocities``,
    ``deformation_gradients`` (n, 3, 3); for the Ding model ``elastic_gradients``,
    ``kirchhoff_stresses`` (n, 3, 3), ``porosities``, ``temperatures`` (n,) and
    ``viscosity_parameter`` (1,); ``young_modulus`` (scalar or (1,)). Returns a dict of the final
    state's arrays (detached copies joined to the autograd graph): the four kinematic arrays and,
    for Ding, ``elastic_gradients``, ``kirchhoff_stresses``, ``porosities``, ``temperatures``.
    The simulator advances by ``steps`` substeps as ``AdvanceUnchecked`` would, and its parameters
    keep the values given. Device flags raised during the run raise ``RuntimeError``.
    """
    unknown = set(inputs) - set(_INPUTS)
    if unknown:
        raise TypeError(f"unknown Rollout inputs: {sorted(unknown)}")
    runner = _Runner(sim, steps, checkpoint_every)
    names = tuple(k for k in _INPUTS if k in inputs)
    values = tuple(inputs[k] for k in names)
    outputs = _RolloutFunction.apply(runner, names, *values)
    keys = [k for k, _ in _KINEMATIC] + ([k for k, _ in _DING] if runner.is_ding else [])
    return dict(zip(keys, outputs))
