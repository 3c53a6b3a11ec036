"""Many independent simulators advanced together under one captured CUDA graph.

Each instance keeps its own state, grid and parameters (different particle counts, grids, oven
temperatures). Two substeps of every instance -- state A -> B and B -> A, which brings the
ping-pong states back -- are captured once into a CUDA graph. ``Advance`` replays the graph: one
host call per two substeps of the whole batch, no per-kernel launch cost.

Small bodies go through device tables of instances (``bk_batch_create``/``bk_batch_substep``):
each stage of the substep is one launch per table, 8-10 launches per substep whatever the number
of bodies. Large bodies launch their own kernels on several streams, so that their kernels and
stages interleave on the GPU (``BatchedSimulators`` below says which body goes where).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .physics.substep import PHASE_MECHANICS, PHASE_TRANSPORT, BkBatchInstance


class BatchedSimulators:
    """Where each instance's kernels come from:

    * ``launch="auto"`` (default): bodies below ``table_particles`` particles go through instance
      tables, larger ones launch their own kernels. Small bodies are launch-bound, and a table steps
      any number of them in 8-10 launches per substep; a large body fills the GPU with its own
      launches, and on separate streams the kernels of different bodies and stages interleave
      (a table launch holds one stage of all its instances, 10-15% slower per kernel than a plain
      launch because every block first copies its instance entry into shared memory).
    * ``launch="table"``: every body through ``groups`` tables (dealt out by particle count so the
      groups weigh about the same), each on a stream of its own.
    * ``launch="streams"``: every body launches its own kernels, spread over ``streams`` streams.
    """

    def __init__(self, simulators, streams=8, launch="auto", groups=2, table_particles=50_000):
        self.sims = list(simulators)
        if not self.sims:
            raise ValueError("no simulators")
        for sim in self.sims:
            if sim.IsSettling:
                raise ValueError("batched simulators must be past settling (settling_duration_s = 0)")
            if sim.retain_history:
                raise ValueError("batched simulators keep no history")
        if launch not in ("auto", "table", "streams"):
            raise ValueError(f"launch must be 'auto', 'table' or 'streams', not {launch!r}")
        self.launch = launch
        self.device = self.sims[0].device
        if launch == "table":
            self.table_sims = list(self.sims)
        elif launch == "streams":
            self.table_sims = []
        else:
            self.table_sims = [s for s in self.sims if s.particle_data.particle_count < table_particles]
        tabled = {id(s) for s in self.table_sims}
        self.stream_sims = [s for s in self.sims if id(s) not in tabled]
        self.groups = max(1, min(int(groups), len(self.table_sims))) if self.table_sims else 0
        count = self.groups + (max(1, int(streams)) if self.stream_sims else 0)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(count)]
        self.graph = None
        self._tables = []       # bk_batch_create handles, one per group
        self._layout = None     # the state pairs (and surrogates) the tables and the graph were made for
        self.particle_count = sum(s.particle_data.particle_count for s in self.sims)

    @staticmethod
    def _substep(sim, state_in, state_out, prescattered=False, prescatter_next=False):
        eng = sim._engine
        ahead = eng.prescatter_allowed()
        eng.run(state_in, state_out, False, PHASE_TRANSPORT | PHASE_MECHANICS, False,
                prescattered=ahead and prescattered, prescatter_next=ahead and prescatter_next,
                accumulate=state_out.transport_state if sim.transport is not None else None)

    def _current_layout(self):
        return tuple((id(sim._current), id(sim.next_state), id(sim._engine.surrogate)) for sim in self.sims)

    def _ensure_layout(self):
        """(Re)build the instance table, and drop a captured graph, when a simulator's ping-pong
        pair or surrogate is not the one they were made for (an odd number of substeps taken
        outside the batch swaps the pair)."""
        layout = self._current_layout()
        if layout == self._layout:
            return
        self.graph = None
        self._free_tables()
        if self.table_sims:
            lib = self.sims[0]._engine.lib
            sims = self.table_sims
            # largest first, each to the lightest group so far
            order = sorted(range(len(sims)), key=lambda k: -sims[k].particle_data.particle_count)
            members, weight = [[] for _ in range(self.groups)], [0] * self.groups
            for k in order:
                g = weight.index(min(weight))
                members[g].append(k)
                weight[g] += sims[k].particle_data.particle_count
            for group in members:
                table = (BkBatchInstance * len(group))()
                for j, k in enumerate(group):
                    sim = sims[k]
                    table[j] = sim._engine.batch_instance(sim._current, sim.next_state)
                handle = ctypes.c_void_p()
                _lib.call_raw(lib.bk_batch_create, "bk_batch_create", table, len(group), ctypes.byref(handle))
                self._tables.append(handle)
        self._layout = layout

    def _free_tables(self):
        for handle in self._tables:
            if handle.value:
                self.sims[0]._engine.lib.bk_batch_destroy(handle)
        self._tables = []

    def __del__(self):
        try:
            self._free_tables()
        except Exception:
            pass

    def _record(self):
        self._ensure_layout()
        main = torch.cuda.current_stream()
        # parity 0 steps every instance A -> B and scatters B's transport fields ahead; parity 1
        # steps B -> A on them
        lib = self.sims[0]._engine.lib
        phases = PHASE_TRANSPORT | PHASE_MECHANICS
        used = []  # only streams forked from `main` join it again (under capture, no other may)
        for table, s in zip(self._tables, self.streams):
            s.wait_stream(main)
            used.append(s)
            with torch.cuda.stream(s):
                stream = _lib.stream_handle()
                for parity, prescattered, ahead in ((0, 0, 1), (1, 1, 0)):
                    _lib.call_raw(lib.bk_batch_substep, "bk_batch_substep", table, parity, phases, prescattered,
                                  ahead, stream)
        own = self.streams[self.groups:]
        for k, sim in enumerate(self.stream_sims):
            s = own[k % len(own)]
            if k < len(own):
                s.wait_stream(main)
                used.append(s)
            with torch.cuda.stream(s):
                a, b = sim._current, sim.next_state
                # the second substep of the pair finds its transport fields scattered by the first
                self._substep(sim, a, b, prescatter_next=True)
                self._substep(sim, b, a, prescattered=True)
        for s in used:
            main.wait_stream(s)

    def capture(self):
        """Build the graph (the simulators' kernels run once outside capture first, to load and
        configure every kernel; that run advances each instance by two substeps)."""
        self._ensure_layout()
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
            if self._current_layout() != self._layout:
                self._ensure_layout()  # drops a graph made for other state pairs
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


class _MappedDoubles:
    """float64 slots in pinned host memory mapped into the device address space (cudaHostAlloc
    with cudaHostAllocMapped): kernels store through ``device_ptr``, the host reads ``view``."""

    def __init__(self, count):
        import ctypes
        import numpy as np
        from cuda.bindings import runtime as cudart
        self._cudart = cudart
        err, self._host_ptr = cudart.cudaHostAlloc(8 * count, cudart.cudaHostAllocMapped)
        if err != cudart.cudaError_t.cudaSuccess:
            raise RuntimeError(f"cudaHostAlloc failed: {err}")
        err, self.device_ptr = cudart.cudaHostGetDevicePointer(self._host_ptr, 0)
        if err != cudart.cudaError_t.cudaSuccess:
            cudart.cudaFreeHost(self._host_ptr)
            raise RuntimeError(f"cudaHostGetDevicePointer failed: {err}")
        self.view = np.ctypeslib.as_array((ctypes.c_double * count).from_address(self._host_ptr))
        self.view[:] = 0.0

    def __del__(self):
        if getattr(self, "_host_ptr", None):
            try:
                self._cudart.cudaFreeHost(self._host_ptr)
            except (TypeError, AttributeError):
                pass  # interpreter shutdown: the runtime bindings are already torn down
            self._host_ptr = None


class StepResult:
    """One substep's (grid mass, kinetic energy), written by its graph into mapped host memory."""

    def __init__(self, event, view):
        self.event = event
        self.view = view

    def get(self):
        """Wait for the substep, then read its two values on the host (no copy is issued). The
        slot is rewritten by the substep two later: read it before launching that one."""
        self.event.synchronize()
        return [float(self.view[0]), float(self.view[1])]


class SubstepGraphs:
    """One simulator's substep as two captured CUDA graphs, state A -> B and B -> A, each followed
    by the step-result reduction (``MpmSimulator.StepSummary``): ``Advance(1)`` is one graph launch.
    For callers that read a result back after every substep, where the per-kernel host launch cost
    would otherwise sit between the substeps.

    ``inputs``: device tensors the caller refills before every substep (per-particle gas source
    rates, say). Each graph starts by copying them from a staging buffer of its own, so ``load``
    can upload the inputs of the substep after the next one from pinned host memory, on a copy
    stream, while the next one runs. ``host_results``: the two graphs write their step results
    into two slots of mapped pinned host memory (the reduction's last kernel stores them there, no
    copy is queued), and ``Advance`` returns a ``StepResult`` for the slot, so a caller can read
    one substep's result while the next one runs. The graphs hold the simulator's arrays and
    parameters at capture time: refill parameter tensors in place between steps, and capture again
    after replacing one.

    ``chained``: each substep's G2P also scatters the next substep's transport fields (volume,
    capacity, energy, water), and each graph uses the fields the previous substep scattered instead
    of running the scalar P2G. Valid while the simulator advances only through this object, with no
    change to the particle state between substeps; ``inputs`` must then be parameters, not state
    arrays (checked)."""

    def __init__(self, sim, inputs=(), host_results=False, chained=False):
        if sim.IsSettling:
            raise ValueError("captured substeps start after settling (settling_duration_s = 0)")
        if sim.retain_history:
            raise ValueError("captured substeps keep no history")
        self.sim = sim
        self.summary = torch.zeros(2, dtype=torch.float64, device=sim.device)
        self._host = None
        if host_results:
            self._host = _MappedDoubles(4)
        self.inputs = list(inputs)
        self.staging = [[torch.empty_like(t) for t in self.inputs] for _ in range(2)]
        self.loaded = [None, None]     # events: staging set k filled
        self.consumed = [None, None]   # events: the last graph that read staging set k finished
        self.graphs = None
        self._first = None
        self.chained = bool(chained) and sim._engine.prescatter_allowed()
        if self.chained:
            state = {t.data_ptr() for st in (sim._current, sim.next_state)
                     for t in _state_tensors_of(st)}
            if any(t.data_ptr() in state for t in self.inputs):
                raise ValueError("chained substeps take parameter inputs only, not particle state arrays")

    def _record(self, state_in, state_out, parity, prescattered=None):
        for t, staged in zip(self.inputs, self.staging[parity]):
            t.copy_(staged)
        chained = self.chained
        BatchedSimulators._substep(self.sim, state_in, state_out,
                                   prescattered=chained if prescattered is None else prescattered,
                                   prescatter_next=chained)
        if self._host is not None:
            self.sim._engine.step_summary(state_out, out_ptr=self._host.device_ptr + 16 * parity)
        else:
            self.sim._engine.step_summary(state_out, self.summary)

    def _parity(self, ahead=0):
        """Staging set read by the substep ``ahead`` substeps after the next one."""
        return ((0 if self.sim._current is self._first else 1) + ahead) % 2

    def capture(self):
        """Build both graphs. The substeps run once outside capture first (which advances the
        simulator by two substeps); the staging buffers then hold the inputs' current values."""
        sim = self.sim
        a, b = sim._current, sim.next_state
        self._first = a
        for k in range(2):
            for t, staged in zip(self.inputs, self.staging[k]):
                staged.copy_(t)
        torch.cuda.synchronize()
        self._record(a, b, 0, prescattered=False)  # the first chained substep scatters its own fields
        self._record(b, a, 1)
        torch.cuda.synchronize()
        sim.step_count += 2
        sim._stale = True
        self._expect_step = sim.step_count
        graphs = {}
        for parity, (src, dst) in enumerate(((a, b), (b, a))):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._record(src, dst, parity)
            graphs[id(src)] = (g, dst, parity)
        self.graphs = graphs
        return self

    def load(self, host_tensors, ahead=0, stream=None):
        """Copy ``host_tensors`` (pinned, one per input) into the staging set of the substep
        ``ahead`` substeps after the next ``Advance`` step, on ``stream`` (default: current)."""
        parity = self._parity(ahead)
        stream = stream or torch.cuda.current_stream()
        with torch.cuda.stream(stream):
            if self.consumed[parity] is not None:
                stream.wait_event(self.consumed[parity])
            for staged, host in zip(self.staging[parity], host_tensors):
                staged.copy_(host, non_blocking=True)
            event = torch.cuda.Event()
            event.record(stream)
        self.loaded[parity] = event

    def Advance(self, steps=1):
        """Advance by ``steps`` substeps. Returns the last one's (grid mass, kinetic energy): a
        device tensor, or with ``host_results`` a ``StepResult``."""
        if self.graphs is None:
            self.capture()
        sim = self.sim
        main = torch.cuda.current_stream()
        for _ in range(steps):
            graph, nxt, parity = self.graphs[id(sim._current)]
            if self.loaded[parity] is not None:
                main.wait_event(self.loaded[parity])
                self.loaded[parity] = None
            if self.chained and sim.step_count != self._expect_step:
                # The simulator was advanced outside this object since the last substep here, so no
                # fields were scattered ahead: this substep runs eagerly with its own scalar P2G.
                self._record(sim._current, nxt, parity, prescattered=False)
            else:
                graph.replay()
            done = torch.cuda.Event()
            done.record(main)
            self.consumed[parity] = done
            sim.next_state, sim._current = sim._current, nxt
            sim.step_count += 1
            sim._stale = True
            self._expect_step = sim.step_count
            if self._host is not None:
                result = StepResult(done, self._host.view[2 * parity:2 * parity + 2])
        return result if self._host is not None and steps > 0 else self.summary


def _state_tensors(sim):
    return _state_tensors_of(sim._current)


def _state_tensors_of(st):
    from dataclasses import fields
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
