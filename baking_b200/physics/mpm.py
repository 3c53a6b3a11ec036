"""MLS-MPM baking simulator (the reference's ``physics/mpm.py:17-340``) on one B200.

Same constructor, attributes and methods as the reference ``MpmSimulator``
(``Step``, ``Advance``, ``Reset``, ``CheckState``, ``UpdateMesh``,
``CaptureSnapshot``/``SaveSnapshot``, the settling state machine), with state in
CUDA tensors and every kernel on the device. Two ping-pong particle states are
allocated once; no array is allocated per substep.

Error flags. ``Step()`` reads the device flags after the transport solve and
after the return map, exactly where the reference synchronises, and raises
before the new state is committed. ``Advance(n)`` runs its substeps without a
host round trip and checks the flags once at the end; a failure then names the
first substep whose flags were set.
"""

from __future__ import annotations

import math
from dataclasses import fields, replace
from pathlib import Path

import numpy as np
import torch

from .. import _lib, arrays
from ..geometry.mesh_tracking import ParticleMeshBinding
from .grid import GridState
from .materials.ding import DingMaterial
from .materials.elastic import ElasticMaterial
from .state import AllocateState, CreateParticleState
from .thermal_water import AllocateTransportState, ThermalWaterTransport



def _plane_layout(t):
    """True for a (n, 3) or (n, 3, 3) view whose components are planes of one pitch."""
    try:
        pitch = arrays.layout_pitch(t)
    except ValueError:
        return False
    if t.dim() == 2:
        return t.stride(0) == 1 and t.stride(1) == pitch
    return t.dim() == 3 and t.stride(0) == 1 and t.stride(2) == pitch and t.stride(1) == 3 * pitch


_DING_SNAPSHOT = ("elastic_gradients", "plastic_gradients", "kirchhoff_stresses", "return_residuals", "porosities",
                  "temperatures", "gelled", "yield_stresses", "viscosities", "gas_moles", "gas_pressures",
                  "porosity_residuals", "reference_densities")


class MpmSimulator:
    def __init__(self, tet_mesh, particle_samples, simulation_config, material_config,
                 initial_velocity=(0.0, 0.0, 0.0), retain_history=False, ding_config=None, transport_config=None,
                 diagnostics="full", sort_interval=0):
        """``diagnostics="full"`` keeps every reference output array current after each substep;
        ``"lean"`` writes only the primary state per substep and fills the derivable arrays
        (plastic gradients, material temperature, density, yield stress, viscosity, gas pressure,
        saturation, particle mass) when ``current_state`` is read. Per-particle return residuals
        are kept only in "full" mode; both modes keep their per-substep maximum.

        ``sort_interval`` k > 0 calls ``SortParticles`` after every k-th substep of ``Step``,
        ``Advance`` and ``AdvanceUnchecked`` (the particle order then changes; 0, the default,
        keeps the sample order)."""
        if diagnostics not in ("full", "lean"):
            raise ValueError("diagnostics must be 'full' or 'lean'")
        if int(sort_interval) != sort_interval or sort_interval < 0 or (sort_interval and retain_history):
            raise ValueError("sort_interval must be a nonnegative integer, and 0 with retain_history")
        self.sort_interval = int(sort_interval)
        self.diagnostics = diagnostics
        simulation_config.Validate(material_config)
        self.device = _lib.require_cuda(simulation_config.device_name)
        self.device_name = str(self.device)
        _lib.load()
        self.tet_mesh = tet_mesh
        self.particle_samples = particle_samples
        self.simulation_config = simulation_config
        self.material = ElasticMaterial(material_config)
        if material_config.model == "ding2019":
            from ..config import DingConfig
            self.material = DingMaterial(material_config, ding_config or DingConfig(), self.device, retain_history)
        if isinstance(self.material, DingMaterial):
            self.material.simulation_config = simulation_config
        if (isinstance(self.material, DingMaterial) and self.material.ding_config.gas_enabled
                and not (transport_config and transport_config.enabled)):
            raise ValueError("Ding gas simulation requires transport.enabled=true; prescribed temperature "
                             "schedules were removed")
        self.initial_velocity = initial_velocity
        self.retain_history = retain_history
        self.ValidateInitialDomain()
        self.mesh_binding = ParticleMeshBinding(tet_mesh, particle_samples, self.device)
        self.transport = None
        self.error_flags = torch.zeros(2, dtype=torch.int32, device=self.device)
        self.error_flags_ding_unused = torch.zeros(3, dtype=torch.int32, device=self.device)
        self.error_flags_transport_unused = torch.zeros(2, dtype=torch.int32, device=self.device)
        if transport_config is not None and transport_config.enabled:
            transport_config.Validate(material_config)
            self.material.initial_temperature_k = transport_config.initial_temperature_k
            self.transport = ThermalWaterTransport(self, transport_config)
        self._buffers = {}
        # particle_order[k]: index in the constructor's samples of the particle at position k
        self.particle_order = torch.arange(len(particle_samples.particle_positions), device=self.device)
        self.sort_count = 0
        # Within one Advance/AdvanceUnchecked call, let each substep's G2P kernel also scatter the
        # next substep's transport fields (one particle pass fewer). Off by default: on the 1M loaf
        # the separate scatter kernel measured 1% faster per substep (2.77e9 against 2.74e9).
        self.scatter_ahead = False
        self.Reset()

    # --------------------------------------------------------------- state
    @property
    def particle_samples(self):
        """The particle samples in the current particle order (permuted on first read after
        SortParticles)."""
        if self._samples_order is not None:
            order = self._samples_order.cpu().numpy()
            s, n = self._particle_samples, len(order)
            self._particle_samples = replace(s, **{
                f.name: np.asarray(getattr(s, f.name))[order] for f in fields(s)
                if np.ndim(getattr(s, f.name)) >= 1 and len(getattr(s, f.name)) == n})
            self._samples_order = None
        return self._particle_samples

    @particle_samples.setter
    def particle_samples(self, samples):
        self._particle_samples = samples
        self._samples_order = None

    @property
    def current_state(self):
        """The accepted state; its derivable reference fields are filled before it is returned."""
        if self._stale:
            self._engine.materialize(self._current, plastic=self.diagnostics == "lean")
            self._stale = False
        return self._current

    @current_state.setter
    def current_state(self, state):
        self._current = state
        self._stale = False

    # ------------------------------------------------------------ settling
    @property
    def settling_steps(self):
        if self.transport is None:
            return 0
        if self._baking_start_step is not None and self._baking_start_step > 0:
            return self._baking_start_step
        return int(math.ceil(self.transport.config.settling_duration_s / self.simulation_config.time_step - 1e-10))

    @property
    def IsSettling(self):
        return (self.transport is not None and self.transport.config.settling_duration_s > 0
                and self._baking_start_step is None)

    @property
    def baking_steps(self):
        return 0 if self.IsSettling else max(0, self.step_count - self.settling_steps)

    @property
    def baking_time(self):
        return self.baking_steps * self.simulation_config.time_step

    def UpdateSettling(self, old_state):
        from .quasistatic import SettlingMetrics
        config = self.transport.config
        dt = self.simulation_config.time_step
        if not config.settling_auto:
            if self.step_count >= self.settling_steps:
                self._baking_start_step = self.step_count
                self.settling_reason = "fixed_duration"
            return
        self.settling_metrics.zero_()
        SettlingMetrics(self.current_state.particle_velocities, self.current_state.affine_velocities,
                        self.settling_reference_plastic, self.current_state.material_state.plastic_gradients,
                        self.settling_metrics, (self.step_count - self.settling_reference_step) * dt)
        values = self.settling_metrics.tolist()
        if (self.step_count - self.settling_reference_step) * dt + 1e-12 >= min(.01, config.settling_hold_duration_s):
            self.settling_plastic_rate = float(values[2])
            self.settling_reference_plastic.copy_(self.current_state.material_state.plastic_gradients)
            self.settling_reference_step = self.step_count
        values[2] = self.settling_plastic_rate
        self.settling_diagnostics = dict(max_speed_m_s=float(values[0]), max_strain_rate_per_s=float(values[1]),
                                         max_plastic_rate_per_s=float(values[2]))
        eligible = (self.step_count - 1) * dt + 1e-12 >= config.settling_min_duration_s
        small = values[0] <= config.settling_speed_tolerance and max(values[1:]) <= config.settling_rate_tolerance
        self.settling_quiet_steps = self.settling_quiet_steps + 1 if eligible and small else 0
        if self.settling_quiet_steps * dt + 1e-12 >= config.settling_hold_duration_s:
            self._baking_start_step = self.step_count
            self.settling_reason = "quasi_static"
        elif self.step_count >= self.settling_steps:
            self.settling_reason = "timeout"
            raise RuntimeError("Settling did not reach quasi-static tolerances before settling_duration_s; "
                               "baking was not started. Increase the maximum duration or review tolerances/material.")

    # -------------------------------------------------------------- set-up
    # ------------------------------------------------------------ particle order
    def CellOrder(self):
        """The permutation that groups the current particles by quadratic stencil base in Morton
        order (``bk_sort_by_cell``, stable): int64 device tensor, position k takes the particle now
        at ``order[k]``."""
        n = self.particle_data.particle_count
        x = self._current.particle_positions
        s = self.simulation_config
        lib = _lib.load()
        need = lib.bk_sort_by_cell_scratch_bytes(n, s.grid_resolution)
        if need < 0:
            raise RuntimeError(f"bk_sort_by_cell_scratch_bytes: {lib.bk_last_error().decode(errors='replace')}")
        scratch = torch.empty(max(int(need), 1), dtype=torch.uint8, device=self.device)
        order = torch.empty(n, dtype=torch.int32, device=self.device)
        origin = (_lib.C.c_float * 3)(*s.grid_origin)
        _lib.call("bk_sort_by_cell", n, arrays.layout_pitch(x) if n else 0, arrays.ptr(x), _lib.C.addressof(origin),
                  s.grid_spacing, s.grid_resolution, order.data_ptr(), scratch.data_ptr(), int(need),
                  _lib.stream_handle())
        return order.long()

    def _particle_arrays(self):
        """Every device array holding one row per particle, each storage view once."""
        n = self.particle_data.particle_count
        out, seen = [], set()

        def visit(t):
            if isinstance(t, torch.Tensor) and t.dim() >= 1 and t.shape[0] == n:
                key = (t.data_ptr(), tuple(t.shape), tuple(t.stride()), t.dtype)
                if key not in seen:
                    seen.add(key)
                    out.append(t)

        def visit_fields(holder):
            if holder is not None:
                for f in fields(holder):
                    visit(getattr(holder, f.name))

        for st in (self._current, self.next_state):
            visit_fields(st)
            visit_fields(st.material_state)
            visit_fields(st.transport_state)
        visit_fields(self.particle_data)
        for t in (self.kirchhoff_stresses, self._stress_water, self.settling_reference_plastic,
                  *self._prepared.values(), *self._buffers.get("transport", {}).values()):
            visit(t)
        if isinstance(self.material, DingMaterial) and n > 1:
            visit(self.material.production_parameter)
        if self.transport is not None:
            for t in (self.transport.reference_volumes, self.transport.dry_masses, self.transport.capacities):
                visit(t)
        return out

    def _permute_arrays(self, order):
        """Every per-particle array in place through bk_permute_particles (arrays gathered in groups
        that fit a scratch buffer of up to 256 MB, or the largest array, two launches per group);
        arrays not in plane layout go through torch."""
        n = self.particle_data.particle_count
        table, largest, total = [], 0, 0
        for t in self._particle_arrays():
            planes = t.numel() // n if n else 0
            pitch = n if t.dim() == 1 else arrays.layout_pitch(t) if _plane_layout(t) else None
            if pitch is None or t.element_size() not in (4, 8) or (t.dim() == 1 and t.stride(0) != 1):
                t.copy_(t.index_select(0, order))
                continue
            table.append(_lib.BkParticleArray(t.data_ptr(), pitch, planes, t.element_size()))
            largest = max(largest, planes * n * t.element_size())
            total += (planes * n * t.element_size() + 255) // 256 * 256
        if not table:
            return
        size = min(total, max(largest, 256 << 20))
        scratch = torch.empty(size, dtype=torch.uint8, device=self.device)
        order32 = order.to(torch.int32)
        entries = (_lib.BkParticleArray * len(table))(*table)
        _lib.call("bk_permute_particles", n, order32.data_ptr(), len(table), _lib.C.addressof(entries),
                  scratch.data_ptr(), size, _lib.stream_handle())

    def SortParticles(self, order=None):
        """Reorder the particles in place by grid cell (``CellOrder``, or a given permutation), so
        that the scatter kernels see long runs of particles sharing a stencil base and compact
        per-block node boxes. No counterpart in the reference, whose kernels read particles in
        sample order; results differ from the unsorted run only by float summation order.

        Every per-particle array (both ping-pong states, constants, gas source rates, settling
        reference) is permuted in place, so captured CUDA graphs stay valid; the particle indices of
        the mesh binding and of the surface face owners are renumbered, and ``particle_samples``
        is replaced by a permuted copy (``Reset`` then starts from the sorted order).
        ``particle_order[k]`` is the index, in the samples given at construction, of the particle
        now at position k. Per-particle inputs given afterwards (gas source rates, rollout inputs)
        are in the new order. Not available while the simulator keeps a state history."""
        if self.retain_history:
            raise ValueError("SortParticles would reorder the kept state history")
        n = self.particle_data.particle_count
        if order is None:
            order = self.CellOrder()
        else:
            order = torch.as_tensor(order, device=self.device).long()
            if order.shape != (n,) or (n and not torch.equal(torch.sort(order).values,
                                                            torch.arange(n, device=self.device))):
                raise ValueError("order must be a permutation of the particle indices")
        if n == 0:
            return order
        self.current_state  # fill the derivable arrays so they move with the particles
        inverse = torch.empty_like(order)
        inverse[order] = torch.arange(n, device=self.device)
        self._permute_arrays(order)
        self.mesh_binding.RenumberParticles(inverse)
        index_arrays = []
        if self.transport is not None:
            index_arrays.append(self.transport.owners)
            surface = getattr(self._engine, "_surface_tensors", None)
            if surface is not None:
                index_arrays.append(surface["owners"])
        for t in index_arrays:
            t.copy_(torch.where(t >= 0, inverse[t.clamp(min=0).long()].to(t.dtype), t))
        # the host samples follow when next read (particle_samples)
        self._samples_order = order if self._samples_order is None else self._samples_order[order]
        self.particle_order = self.particle_order[order]
        self.sort_count += 1
        self._buffers.pop("rollout", None)  # reverse-mode buffers hold per-particle copies
        self._stale = True
        return order

    def SetGasSourceRates(self, rates):
        """Per-particle gas source rate alpha_i (mol/(kg s)) in place of the scalar production parameter."""
        rates = torch.as_tensor(np.asarray(rates, dtype=np.float32), device=self.device).reshape(-1)
        if rates.shape[0] not in (1, self.particle_data.particle_count):
            raise ValueError("gas source rates need one value or one per particle")
        self.material.production_parameter = rates.contiguous()

    def Masses(self, state=None):
        state = self.current_state if state is None else state
        return state.transport_state.particle_masses if state.transport_state is not None else \
            self.particle_data.particle_masses

    def ValidateInitialDomain(self):
        s = self.simulation_config
        origin = np.asarray(s.grid_origin)
        lower = origin + (s.boundary_cells - 1) * s.grid_spacing
        upper = origin + (s.grid_resolution - s.boundary_cells) * s.grid_spacing
        points = np.concatenate([self.tet_mesh.vertex_positions, self.particle_samples.particle_positions])
        if np.any(points < lower) or np.any(points > upper):
            raise ValueError(f"model must initially fit inside {lower} .. {upper}; adjust [mesh] mesh_scale/"
                             "mesh_translation or [simulation] grid settings in the config file")

    def surface_vertices_buffer(self):
        if "vertices" not in self._buffers:
            self._buffers["vertices"] = arrays.vec3s(len(self.tet_mesh.vertex_positions), device=self.device)
        return self._buffers["vertices"]

    def transport_particle_workspace(self):
        if "transport" not in self._buffers:
            n = self.particle_data.particle_count
            self._buffers["transport"] = {name: arrays.scalars(n, torch.float64, self.device)
                                          for name in ("exposed", "contact", "particle_heat", "particle_loss")}
        return self._buffers["transport"]

    def _allocate_like_current(self, share_accumulators=True):
        n = self.particle_data.particle_count
        state = AllocateState(n, self.device)
        if isinstance(self.material, DingMaterial):
            self.material.InitializeState(state)
        if self.transport is not None:
            state.transport_state = AllocateTransportState(n, self.device)
            current = self._current.transport_state
            if share_accumulators:
                # Loss/exchange only change for face-owning particles; both ping-pong states share them.
                state.transport_state.water_losses = current.water_losses
                state.transport_state.heat_exchanges = current.heat_exchanges
            else:
                state.transport_state.water_losses = current.water_losses.clone()
                state.transport_state.heat_exchanges = current.heat_exchanges.clone()
        return state

    def Reset(self):
        self._buffers.pop("rollout", None)  # reverse-mode buffers belong to the previous engine
        if isinstance(self.material, DingMaterial):
            self.material.Reset()
        self._stale = False
        self._current, self.particle_data = CreateParticleState(self.particle_samples, self.device,
                                                                self.initial_velocity, self.retain_history)
        if isinstance(self.material, DingMaterial):
            self.material.InitializeState(self._current)
        if self.transport is not None:
            self.transport.InitializeState(self._current)
        self.next_state = self._allocate_like_current()
        n = self.particle_data.particle_count
        self.grid_state = GridState(self.simulation_config, self.device)
        self.kirchhoff_stresses = arrays.mat33s(n, device=self.device)
        self._stress_water = arrays.mat33s(n, device=self.device)
        self._prepared = dict(temperatures=arrays.scalars(n, torch.float32, self.device),
                              reference_densities=arrays.scalars(n, torch.float32, self.device),
                              saturations=arrays.scalars(n, torch.float64, self.device),
                              gas_moles=arrays.scalars(n, torch.float64, self.device),
                              gas_pressures=arrays.scalars(n, torch.float64, self.device))
        self.vertex_positions = arrays.from_numpy(self.tet_mesh.vertex_positions.astype(np.float32), "f4",
                                                  self.device)
        self.error_flags.zero_()
        if self.transport is not None:
            self.transport.error_flags.zero_()
        self.state_history = [self.current_state] if self.retain_history else []
        self.workspace_history = []
        self.transport_workspace_history = []
        self.step_count = 0
        self._baking_start_step = None if (self.transport is not None
                                           and self.transport.config.settling_duration_s > 0) else 0
        self.settling_quiet_steps = 0
        self.settling_reference_step = 0
        self.settling_plastic_rate = 0.0
        self.settling_reference_plastic = None
        if isinstance(self.material, DingMaterial):
            # A plane-layout copy: bk_settling_metrics reads it with the state's pitch (a clone of
            # the strided view would be row-major unless n fills the pitch).
            plastic = self.current_state.material_state.plastic_gradients
            self.settling_reference_plastic = arrays.mat33s(n, device=self.device, pitch=arrays.layout_pitch(plastic))
            self.settling_reference_plastic.copy_(plastic)
        self.settling_reason = "pending" if self._baking_start_step is None else "disabled"
        self.settling_diagnostics = dict(max_speed_m_s=0.0, max_strain_rate_per_s=0.0, max_plastic_rate_per_s=0.0)
        self.settling_metrics = torch.zeros(3, dtype=torch.float32, device=self.device)
        self.mesh_step_count = 0
        from .substep import SubstepEngine
        self._engine = SubstepEngine(self)
        if getattr(self, "result_recorder", None) is not None:
            self.result_recorder.Reset()

    # ---------------------------------------------------------------- step
    def _substep(self, check, prescattered=False, prescatter_next=False):
        """One substep through the fused kernels; with ``check`` the device flags are read where the
        reference synchronises (after the transport solve and after the return map).
        ``prescattered``/``prescatter_next``: the transport fields of this substep were scattered
        ahead by the previous one / scatter the next substep's ahead (SubstepEngine.run); only for
        substeps run back to back inside one call, where nothing can change the state in between."""
        from .substep import PHASE_MECHANICS, PHASE_TRANSPORT
        was_settling = self.IsSettling
        original = self._current
        output = self._allocate_like_current(share_accumulators=False) if self.retain_history else self.next_state
        full = self.diagnostics == "full"
        if check and self.transport is not None:
            self._engine.run(original, output, was_settling, PHASE_TRANSPORT, full, prescattered=prescattered)
            self.transport.CheckState()
            self._engine.run(original, output, was_settling, PHASE_MECHANICS, full, prescatter_next=prescatter_next)
        else:
            # unchecked: the surface kernel advances the accumulators (nothing can reject the substep)
            self._engine.run(original, output, was_settling, PHASE_TRANSPORT | PHASE_MECHANICS, full,
                             prescattered=prescattered, prescatter_next=prescatter_next,
                             accumulate=output.transport_state if self.transport is not None else None)
        if check and isinstance(self.material, DingMaterial):
            self.material.CheckState()
        if check and self.transport is not None:
            self._engine.accumulate_surface(output.transport_state)
        if self.retain_history:
            self.state_history.append(output)
        self._current = output
        self.next_state = original
        self._stale = True
        if full:
            self._engine.materialize(output, plastic=False)
            self._stale = False
        self.step_count += 1
        if was_settling:
            self.UpdateSettling(original)
        if getattr(self, "result_recorder", None) is not None:
            self.result_recorder.Record()
            if was_settling and not self.IsSettling:
                self.result_recorder.settled_measurement = dict(self.result_recorder.last_measurement)
                self.result_recorder.QueueSnapshot()
        if self.sort_interval and self.step_count % self.sort_interval == 0:
            self.SortParticles()

    def MaxReturnResiduals(self):
        """(max return residual, max porosity residual) of the last substep, on the host."""
        return tuple(self._engine.max_residuals.tolist())

    def Step(self):
        self._substep(check=True)

    def _device_flag_messages(self):
        messages = []
        if isinstance(self.material, DingMaterial):
            m = self.material.FlagMessage(self.material.error_flags.tolist())
            if m:
                messages.append(m)
        if self.transport is not None:
            m = self.transport.FlagMessage(self.transport.error_flags.tolist())
            if m:
                messages.append(m)
        return messages

    def Advance(self, step_count):
        if step_count < 1:
            raise ValueError("step_count must be positive")
        start = self.step_count
        ahead = self.scatter_ahead and self._engine.prescatter_allowed()
        for k in range(step_count):
            self._substep(check=self.IsSettling, prescattered=ahead and k > 0,
                          prescatter_next=ahead and k + 1 < step_count)
        values = self._check_values()
        messages = []
        if isinstance(self.material, DingMaterial):
            m = self.material.FlagMessage([values["ding_flag0"], values["ding_flag1"], values["ding_flag2"]])
            if m:
                messages.append(m)
        if self.transport is not None:
            m = self.transport.FlagMessage([values["transport_flag0"], values["transport_flag1"]])
            if m:
                messages.append(m)
        if messages:
            raise RuntimeError(messages[0] + f" (flag raised within substeps {start + 1}..{self.step_count})")
        return self.CheckState(values)

    def AdvanceUnchecked(self, step_count):
        """Run substeps with no host synchronisation; flags stay on the device until CheckState/Advance.
        With ``scatter_ahead`` set, each substep's G2P within the call scatters the next substep's
        transport fields ahead."""
        ahead = self.scatter_ahead and self._engine.prescatter_allowed()
        for k in range(step_count):
            self._substep(check=False, prescattered=ahead and k > 0, prescatter_next=ahead and k + 1 < step_count)

    def StepSummary(self, out=None):
        """Device tensor (grid mass of the last substep, particle kinetic energy of the current
        state), float64, from one fused reduction (``bk_step_summary``); ``out`` (2 doubles) may
        be given to write into."""
        return self._engine.step_summary(self._current, out)

    def AlgorithmicBytes(self, kernel, active_nodes):
        """Bytes one launch of ``kernel`` must move (each input and output array once), or None."""
        from ..roofline import algorithmic_bytes
        return algorithmic_bytes(kernel, self, active_nodes)

    def UpdateMesh(self, force_update=False):
        if force_update or self.mesh_step_count != self.step_count:
            self.mesh_binding.Reconstruct(self.current_state, self.vertex_positions)
            self.mesh_step_count = self.step_count

    def _check_values(self):
        """Every input of CheckState from one device reduction over the current state, the mesh
        vertices and the grid (bk_check_state), read back in one small copy."""
        self.UpdateMesh()
        return self._engine.check_state(self._current)

    def CheckState(self, values=None):
        """physics/mpm.py:243-308: the same checks, messages and returned summary. ``values`` are the
        reduction's results when the caller already has them (Advance)."""
        v = self._check_values() if values is None else values
        if v["substep_status"]:
            raise RuntimeError("a substep kernel gave up waiting for a device copy or tensor-core result; "
                               "its particles were left unprocessed")
        if v["sim_flag0"]:
            raise RuntimeError("nonpositive/nonfinite J; reduce dt or inspect loading and sampling")
        if v["sim_flag1"]:
            raise RuntimeError("particle stencil left the grid; enlarge the domain or reduce dt")
        if v["nonfinite_state"]:
            raise RuntimeError("nonfinite particle state; simulation stopped")
        if v["j_min"] <= 0.0:
            raise RuntimeError("inverted particle deformation; reduce dt or loading")
        if v["outside_stencil"]:
            raise RuntimeError("particle outside valid grid stencil")
        sim = self.simulation_config
        vmax = v["speed_max"]
        wave = self.material.material_config.wave_speed
        if isinstance(self.material, DingMaterial) and self.material.ding_config.gas_enabled:
            wave = max(wave, v["gas_wave_max"])
        if self.transport is not None and self.transport.config.water_enabled:
            wave = float(math.sqrt(wave * wave + v["water_wave2_max"]))
        cfl = (vmax + wave) * sim.time_step / sim.grid_spacing
        if cfl > sim.cfl_limit:
            raise RuntimeError(f"estimated CFL={cfl:.3f} > {sim.cfl_limit}; reduce dt")
        if isinstance(self.material, DingMaterial):
            message = self.material.FlagMessage([v["ding_flag0"], v["ding_flag1"], v["ding_flag2"]])
            if message:
                raise RuntimeError(message)
            if v["nonfinite_ding"]:
                raise RuntimeError("nonfinite Ding internal state")
            if v["residual_max"] > 1e-4:
                raise RuntimeError("Ding local return mapping did not converge")
        if v["nonfinite_vertices"]:
            raise RuntimeError("nonfinite reconstructed mesh vertices")
        return {
            "step_count": self.step_count,
            "simulation_time": self.step_count * sim.time_step,
            "particle_count": self.particle_data.particle_count,
            "particle_volume_m3": v["particle_volume"],
            "total_mass": v["total_mass"],
            "grid_mass": v["grid_mass"],
            "minimum_j": v["j_min"],
            "maximum_j": v["j_max"],
            "maximum_speed": vmax,
            "kinetic_energy": v["kinetic_energy"],
            "estimated_cfl": cfl,
            "unmapped_mesh_vertices": self.mesh_binding.unmapped_vertex_count,
            "inverted_mesh_tets": int(v["inverted_tets"]),
        }

    # ------------------------------------------------------------ snapshots
    def CaptureSnapshot(self):
        self.UpdateMesh()
        st = self.current_state
        snap = dict(
            particle_positions=arrays.to_numpy(st.particle_positions).copy(),
            particle_velocities=arrays.to_numpy(st.particle_velocities).copy(),
            deformation_gradients=arrays.to_numpy(st.deformation_gradients).copy(),
            affine_velocities=arrays.to_numpy(st.affine_velocities).copy(),
            particle_masses=arrays.to_numpy(self.Masses()).copy(),
            reference_volumes=arrays.to_numpy(self.particle_data.reference_volumes).copy(),
            vertices=arrays.to_numpy(self.vertex_positions).copy(), tetrahedra=self.tet_mesh.tet_indices.copy(),
            reference_vertices=self.tet_mesh.vertex_positions.copy(),
            source_tets=np.asarray(self.particle_samples.source_tets).copy(),
            simulation_time=self.step_count * self.simulation_config.time_step,
            baking_time_s=self.baking_time, settling_steps=self.settling_steps)
        if self.sort_count:
            snap["particle_order"] = self.particle_order.cpu().numpy()  # after SortParticles
        if isinstance(self.material, DingMaterial):
            for name in _DING_SNAPSHOT:
                snap["ding_" + name] = arrays.to_numpy(getattr(st.material_state, name)).copy()
        if st.transport_state is not None:
            for field in fields(st.transport_state):
                snap["transport_" + field.name] = arrays.to_numpy(getattr(st.transport_state, field.name)).copy()
        # Resume fields (LoadSnapshot; the reference writes no resume data): the step counter, the
        # settling state machine and the per-particle gas source rates.
        snap.update(resume_step_count=self.step_count, resume_mesh_step_count=self.mesh_step_count,
                    resume_baking_start_step=-1 if self._baking_start_step is None else self._baking_start_step,
                    resume_settling_quiet_steps=self.settling_quiet_steps,
                    resume_settling_reference_step=self.settling_reference_step,
                    resume_settling_plastic_rate=self.settling_plastic_rate,
                    resume_settling_reason=self.settling_reason)
        if self.settling_reference_plastic is not None:
            snap["resume_settling_reference_plastic"] = arrays.to_numpy(self.settling_reference_plastic).copy()
        if isinstance(self.material, DingMaterial):
            snap["resume_gas_source_rates"] = self.material.production_parameter.cpu().numpy().copy()
        return snap

    def LoadSnapshot(self, snapshot):
        """Resume from a snapshot (a path written by ``SaveSnapshot`` or a ``CaptureSnapshot``
        dict) of a simulator built from the same scene and configuration. Restores the particle
        state, the mesh vertices, the step counter, the settling state machine, the gas source
        rates and, for a sorted simulator, its particle order; the next substep continues the
        saved run (up to float summation order). The reference saves snapshots but cannot load
        them."""
        if isinstance(snapshot, (str, Path)):
            with np.load(snapshot) as data:
                snap = {k: data[k] for k in data.files}
        else:
            snap = dict(snapshot)
        if self.retain_history:
            raise ValueError("LoadSnapshot would bypass the kept state history")
        if "resume_step_count" not in snap:
            raise ValueError("the snapshot has no resume fields")
        n = self.particle_data.particle_count
        if (len(snap["particle_positions"]) != n or not np.array_equal(snap["tetrahedra"], self.tet_mesh.tet_indices)
                or abs(float(snap["simulation_time"]) - int(snap["resume_step_count"]) *
                       self.simulation_config.time_step) > 1e-9 * max(1.0, float(snap["simulation_time"]))):
            raise ValueError("the snapshot belongs to another scene or time step")
        order = snap.get("particle_order")
        current = self.particle_order.cpu().numpy()
        target = np.arange(n) if order is None else np.asarray(order)
        if not np.array_equal(target, current):
            inverse = np.empty(n, dtype=np.int64)
            inverse[current] = np.arange(n)
            self.SortParticles(order=inverse[target])
        if not np.array_equal(snap["reference_volumes"], arrays.to_numpy(self.particle_data.reference_volumes)):
            raise ValueError("the snapshot's reference volumes differ from this simulator's")
        st = self._current
        for name in ("particle_positions", "particle_velocities", "deformation_gradients", "affine_velocities"):
            arrays.assign(getattr(st, name), snap[name])
        if isinstance(self.material, DingMaterial):
            for name in _DING_SNAPSHOT:
                arrays.assign(getattr(st.material_state, name), snap["ding_" + name])
            rates = snap.get("resume_gas_source_rates")
            if rates is not None:
                if rates.shape == tuple(self.material.production_parameter.shape):
                    arrays.assign(self.material.production_parameter, rates)
                else:
                    self.SetGasSourceRates(rates)
        if st.transport_state is not None:
            for field in fields(st.transport_state):
                arrays.assign(getattr(st.transport_state, field.name), snap["transport_" + field.name])
        arrays.assign(self.vertex_positions, snap["vertices"])
        if self.settling_reference_plastic is not None and "resume_settling_reference_plastic" in snap:
            arrays.assign(self.settling_reference_plastic, snap["resume_settling_reference_plastic"])
        self.step_count = int(snap["resume_step_count"])
        self.mesh_step_count = int(snap["resume_mesh_step_count"])
        start = int(snap["resume_baking_start_step"])
        self._baking_start_step = None if start < 0 else start
        self.settling_quiet_steps = int(snap["resume_settling_quiet_steps"])
        self.settling_reference_step = int(snap["resume_settling_reference_step"])
        self.settling_plastic_rate = float(snap["resume_settling_plastic_rate"])
        self.settling_reason = str(snap["resume_settling_reason"])
        self.error_flags.zero_()
        if self.transport is not None:
            self.transport.error_flags.zero_()
        if isinstance(self.material, DingMaterial):
            self.material.error_flags.zero_()
        self._buffers.pop("rollout", None)
        self._stale = True

    def SaveSnapshot(self, output_path):
        self.UpdateMesh()
        output_path = Path(output_path)
        output_path.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(output_path, **self.CaptureSnapshot())
