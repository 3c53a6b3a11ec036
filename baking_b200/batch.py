"""Many independent simulators advanced together under one captured CUDA graph.

Each instance keeps its own state, grid and parameters (different particle counts, grids, oven
temperatures). Two substeps of every instance -- state A -> B and B -> A, which brings the
ping-pong states back -- are captured once into a CUDA graph, instances spread over several
streams so that the kernels of small bodies run side by side on the GPU. ``Advance`` replays
the graph: one host call per two substeps of the whole batch, no per-kernel launch cost.
"""
from __future__ import annotations

import torch

from . import _lib
from .physics.substep import PHASE_MECHANICS, PHASE_TRANSPORT


class BatchedSimulators:
    def __init__(self, simulators, streams=8):
        self.sims = list(simulators)
        if not self.sims:
            raise ValueError("no simulators")
        for sim in self.sims:
            if sim.IsSettling:
                raise ValueError("batched simulators must be past settling (settling_duration_s = 0)")
            if sim.retain_history:
                raise ValueError("batched simulators keep no history")
        self.device = self.sims[0].device
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, int(streams)))]
        self.graph = None
        self.particle_count = sum(s.particle_data.particle_count for s in self.sims)

    @staticmethod
    def _substep(sim, state_in, state_out):
        eng = sim._engine
        eng.run(state_in, state_out, False, PHASE_TRANSPORT | PHASE_MECHANICS, False)
        if sim.transport is not None:
            eng.accumulate_surface(state_out.transport_state)

    def _record(self):
        main = torch.cuda.current_stream()
        for k, sim in enumerate(self.sims):
            s = self.streams[k % len(self.streams)]
            s.wait_stream(main)
            with torch.cuda.stream(s):
                a, b = sim._current, sim.next_state
                self._substep(sim, a, b)
                self._substep(sim, b, a)
        for s in self.streams:
            main.wait_stream(s)

    def capture(self):
        """Build the graph (the simulators' kernels run once outside capture first, to load and
        configure every kernel; that run advances each instance by two substeps)."""
        torch.cuda.synchronize()
        self._record()
        torch.cuda.synchronize()
        self._advance_counters(2)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._record()
        return self

    def _advance_counters(self, steps):
        for sim in self.sims:
            sim.step_count += steps
            sim._stale = True

    def Advance(self, steps, graph=True):
        """Advance every instance by ``steps`` (even) substeps; with ``graph=False`` the same
        kernels are launched one by one (the comparison without the graph)."""
        if steps % 2:
            raise ValueError("steps must be even (the graph holds a pair of ping-pong substeps)")
        if graph:
            if self.graph is None:
                self.capture()
            for _ in range(steps // 2):
                self.graph.replay()
        else:
            for _ in range(steps // 2):
                self._record()
        self._advance_counters(steps)

    def CheckState(self):
        """Each instance's CheckState (device flags, finiteness, CFL) after the last replay."""
        return [sim.CheckState() for sim in self.sims]


def _state_tensors(sim):
    from dataclasses import fields
    st = sim._current
    out = []
    for holder in (st, st.material_state, st.transport_state):
        if holder is None:
            continue
        for f in fields(holder):
            v = getattr(holder, f.name)
            if isinstance(v, torch.Tensor):
                out.append(v)
    return out


def SnapshotStates(sims):
    """Copies of every state array of each simulator's current state."""
    return [[t.clone() for t in _state_tensors(sim)] for sim in sims]


def RestoreStates(sims, snapshot):
    """Put back the arrays taken by SnapshotStates (same simulators, same current states)."""
    for sim, saved in zip(sims, snapshot):
        for t, v in zip(_state_tensors(sim), saved):
            t.copy_(v)
        sim._stale = True
