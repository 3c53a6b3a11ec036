"""Host side of the fused substep (``bk_substep``/``bk_materialize`` in the C ABI).

Builds the pointer structs of ``include/baking_b200.h`` from a simulator's
tensors and launches one substep, or the two halves of one (transport, then
mechanics) when the caller checks the device flags in between.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib, arrays
from ..surrogate import BkMlpNorm
from .materials.ding import DingMaterial, ding_params
from .thermal_water import scalar_params

P = C.c_void_p


class BkState(C.Structure):
    _fields_ = [("x", P), ("v", P), ("C", P), ("F", P), ("Fe", P), ("tau", P), ("porosity", P), ("gelled", P),
                ("material_temperature", P), ("temperature", P), ("water", P), ("gas_moles", P)]


class BkConstants(C.Structure):
    _fields_ = [("volume", P), ("mass", P), ("capacity", P), ("dry_mass", P), ("gas_rate", P),
                ("gas_rate_per_particle", C.c_int32), ("viscosity_parameter", P), ("heat_parameter", P)]


class BkGrid(C.Structure):
    _fields_ = [("node_pm", P), ("node_v", P), ("fields", P * 7), ("node_dT_ratio", P), ("bounds", P)]


class BkSurface(C.Structure):
    _fields_ = [("vertex_count", C.c_int64), ("vertex_ids", P), ("binding_offsets", P), ("binding_particles", P),
                ("binding_weights", P), ("binding_pitch", C.c_int64), ("reference_offsets", P),
                ("vertex_pitch", C.c_int64), ("vertices", P), ("reference_vertices", P), ("owner_count", C.c_int64),
                ("owners", P), ("owner_face_offsets", P), ("faces", P), ("owner_heat", P), ("owner_loss", P),
                ("floor_height", C.c_float), ("contact_distance", C.c_float), ("binding_count", C.c_int64),
                ("accumulate_water_losses", P), ("accumulate_heat_exchanges", P), ("accumulate_time_step", C.c_float)]


class BkDiagnostics(C.Structure):
    _fields_ = [("plastic_gradients", P), ("return_residuals", P), ("porosity_residuals", P), ("max_residuals", P)]


class BkFlags(C.Structure):
    _fields_ = [("simulation", P), ("ding", P), ("transport", P)]


class BkReturnSurrogate(C.Structure):
    _fields_ = [("packed", P), ("norm", BkMlpNorm), ("in_low", C.c_float * 8), ("in_high", C.c_float * 8),
                ("samples", P), ("sample_count", P), ("sample_capacity", C.c_int32), ("sample_stride", C.c_int32),
                ("sample_offset", C.c_int32), ("judge_error", P), ("judge_stride", C.c_int32), ("path_counts", P)]


class BkSubstepParams(C.Structure):
    _fields_ = [("n", C.c_int64), ("pitch", C.c_int64), ("resolution", C.c_int32), ("boundary_cells", C.c_int32),
                ("origin", C.c_float * 3), ("spacing", C.c_float), ("time_step", C.c_float),
                ("gravity", C.c_float * 3), ("material", C.c_int32), ("ding", _lib.BkDingParams),
                ("transport", C.c_int32), ("gas", C.c_int32), ("settling", C.c_int32), ("scalar", _lib.BkScalarParams),
                ("conductivity", C.c_float), ("diffusivity", C.c_float), ("initial_saturation", C.c_float),
                ("water_stress", C.c_float), ("gas_ambient_pressure", C.c_float), ("density", C.c_float),
                ("elastic_modulus", C.c_float), ("cfl_limit", C.c_float), ("gas_peak", C.c_float),
                ("gas_width", C.c_float), ("surrogate", C.POINTER(BkReturnSurrogate)),
                ("keep_transport_fields", C.c_int32), ("transport_prescattered", C.c_int32),
                ("transport_prescatter_next", C.c_int32), ("transport_prescatter_stale", C.c_int32),
                ("status", P)]


PHASE_TRANSPORT = 1
PHASE_MECHANICS = 2


class BkBatchInstance(C.Structure):
    _fields_ = [("params", BkSubstepParams), ("states", BkState * 2), ("water_losses", P * 2),
                ("heat_exchanges", P * 2), ("constants", BkConstants), ("grid", BkGrid), ("surface", BkSurface),
                ("diagnostics", BkDiagnostics), ("flags", BkFlags)]


class BkCheckInputs(C.Structure):
    _fields_ = [("n", C.c_int64), ("pitch", C.c_int64), ("x", P), ("v", P), ("F", P), ("C", P),
                ("reference_volume", P), ("mass", P), ("dry_mass", P), ("water", P), ("temperature", P),
                ("material_temperature", P), ("Fe", P), ("porosity", P), ("gas_moles", P),
                ("return_residuals", P), ("max_residuals", P), ("sim_flags", P), ("ding_flags", P),
                ("transport_flags", P), ("origin", C.c_float * 3), ("spacing", C.c_float),
                ("resolution", C.c_int32), ("water_enabled", C.c_int32), ("density", C.c_float),
                ("water_density", C.c_float), ("water_stress", C.c_float), ("gas_modulus", C.c_float),
                ("initial_porosity", C.c_float), ("node_pm", P), ("box", P), ("vertex_count", C.c_int64),
                ("vertex_pitch", C.c_int64), ("vertices", P), ("tet_count", C.c_int64), ("tets", P),
                ("substep_status", P)]


# Slots of bk_check_state (include/baking_b200.h, BK_CHECK_*).
CHECK_SLOTS = ("sim_flag0", "sim_flag1", "ding_flag0", "ding_flag1", "ding_flag2", "transport_flag0",
               "transport_flag1", "nonfinite_state", "j_min", "j_max", "outside_stencil", "speed_max", "gas_wave_max",
               "water_wave2_max", "nonfinite_ding", "residual_max", "particle_volume", "total_mass", "kinetic_energy",
               "grid_mass", "nonfinite_vertices", "inverted_tets", "substep_status")
CHECK_BLOCKS = 296

_SIGS = {
    "bk_check_state": [P, P, P, P],
    "bk_substep": [P] * 8 + [C.c_int32, P],
    "bk_materialize": [P] * 11 + [P],
    "bk_surface_accumulate": [P, C.c_float, P, P, P],
    "bk_batch_create": [P, C.c_int32, P],
    "bk_batch_substep": [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P],
    "bk_batch_destroy": [P],
}


def _declare():
    lib = _lib.load()
    for name, argtypes in _SIGS.items():
        fn = getattr(lib, name)
        if fn.argtypes != argtypes:
            fn.restype = C.c_int
            fn.argtypes = argtypes
    return lib


def _p(t):
    return None if t is None else t.data_ptr()


def state_struct(state, material_is_ding, transport, gas):
    s = BkState()
    s.x, s.v = _p(state.particle_positions), _p(state.particle_velocities)
    s.C, s.F = _p(state.affine_velocities), _p(state.deformation_gradients)
    if material_is_ding:
        m = state.material_state
        s.Fe, s.tau = _p(m.elastic_gradients), _p(m.kirchhoff_stresses)
        s.porosity, s.gelled, s.material_temperature = _p(m.porosities), _p(m.gelled), _p(m.temperatures)
        if gas:
            s.gas_moles = _p(m.gas_moles)
    if transport:
        t = state.transport_state
        s.temperature, s.water = _p(t.temperatures), _p(t.water_masses)
    return s


class SubstepEngine:
    """Launches the fused substep for one ``MpmSimulator``."""

    def __init__(self, sim):
        self.sim = sim
        self.lib = _declare()
        dev = sim.device
        s = sim.simulation_config
        R = s.grid_resolution
        self.is_ding = isinstance(sim.material, DingMaterial)
        self.transport = sim.transport is not None
        self.gas = bool(self.is_ding and sim.material.ding_config.gas_enabled)
        n = sim.particle_data.particle_count
        self.n = n
        self.pitch = arrays.layout_pitch(sim._current.deformation_gradients)
        # The grid state's momentum/velocity nodes hold the last substep; the transport fields are
        # zero between substeps. The kernels keep both invariants over the active node boxes.
        sim.grid_state.Clear()
        self.node_pm = sim.grid_state.node_pm
        self.node_v = sim.grid_state.node_v
        self.fields = [torch.zeros(R ** 3 if self.transport else 1, dtype=torch.float64, device=dev)
                       for _ in range(7)]
        self.node_dT_ratio = torch.zeros(R ** 3 if self.transport else 1, 2, dtype=torch.float64, device=dev)
        empty = [2 ** 31 - 1] * 3 + [-2 ** 31] * 3
        # the substep's box, the previous substep's, the transport box scattered ahead
        self.bounds = torch.tensor(empty + empty + empty, dtype=torch.int32, device=dev)
        self.grid = BkGrid()
        self.grid.node_pm, self.grid.node_v = _p(self.node_pm), _p(self.node_v)
        for k in range(7):
            self.grid.fields[k] = _p(self.fields[k])
        self.grid.node_dT_ratio, self.grid.bounds = _p(self.node_dT_ratio), _p(self.bounds)
        self.max_residuals = torch.zeros(2, dtype=torch.float32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)  # BkSubstepParams.status
        # True while the simulator's own grid holds transport fields scattered ahead that no substep
        # has used yet (the last substep run on it had prescatter_next, or a chained graph did).
        self.prescatter_pending = False
        self.surface = BkSurface()
        if self.transport:
            self._build_surface()
        # Return-map surrogate or sample harvest (BkReturnSurrogate), None for the exact map.
        self.surrogate = None
        self.flags = BkFlags()
        self.flags.simulation = _p(sim.error_flags)
        self.flags.ding = _p(sim.material.error_flags) if self.is_ding else _p(sim.error_flags_ding_unused)
        self.flags.transport = _p(sim.transport.error_flags) if self.transport else _p(sim.error_flags_transport_unused)

    # ------------------------------------------------------------------ setup
    def _build_surface(self):
        sim, dev = self.sim, self.sim.device
        tr = sim.transport
        faces = tr.faces.cpu().numpy()
        owners = tr.owners.cpu().numpy()
        order = np.argsort(owners, kind="stable")
        owner_ids, starts = np.unique(owners[order], return_index=True)
        offsets = np.concatenate([starts, [len(order)]]).astype(np.int32)
        self._surface_tensors = dict(
            vertex_ids=torch.as_tensor(np.unique(faces).astype(np.int32), device=dev),
            owners=torch.as_tensor(owner_ids.astype(np.int32), device=dev),
            owner_face_offsets=torch.as_tensor(offsets, device=dev),
            faces=torch.as_tensor(np.ascontiguousarray(faces[order]).astype(np.int32), device=dev),
            owner_heat=torch.zeros(len(owner_ids), dtype=torch.float64, device=dev),
            owner_loss=torch.zeros(len(owner_ids), dtype=torch.float64, device=dev))
        t = self._surface_tensors
        mb = sim.mesh_binding
        sf = self.surface
        sf.vertex_count = int(t["vertex_ids"].shape[0])
        sf.vertex_ids = _p(t["vertex_ids"])
        sf.binding_offsets = _p(mb.binding_offsets)
        sf.binding_particles = _p(mb.binding_particles)
        sf.binding_weights = _p(mb.binding_weights)
        sf.binding_pitch = arrays.layout_pitch(mb.reference_offsets)
        sf.reference_offsets = _p(mb.reference_offsets)
        verts = sim.surface_vertices_buffer()
        sf.vertex_pitch = arrays.layout_pitch(verts)
        if arrays.layout_pitch(mb.reference_vertices) != sf.vertex_pitch:
            raise RuntimeError("vertex arrays must share a plane pitch")
        sf.vertices = _p(verts)
        sf.reference_vertices = _p(mb.reference_vertices)
        sf.owner_count = int(t["owners"].shape[0])
        sf.owners, sf.owner_face_offsets, sf.faces = _p(t["owners"]), _p(t["owner_face_offsets"]), _p(t["faces"])
        sf.owner_heat, sf.owner_loss = _p(t["owner_heat"]), _p(t["owner_loss"])
        ids = t["vertex_ids"].cpu().numpy()
        offs = mb.tables.binding_offsets
        self.surface_bindings = int((offs[ids + 1] - offs[ids]).sum())
        sf.binding_count = self.surface_bindings
        self.owned_faces = int(len(faces))
        s = sim.simulation_config
        sf.floor_height = s.grid_origin[1] + (s.boundary_cells - 1) * s.grid_spacing
        sf.contact_distance = tr.config.contact_distance

    def params(self, settling):
        sim = self.sim
        s = sim.simulation_config
        mc = sim.material.material_config
        p = BkSubstepParams()
        p.n, p.pitch = self.n, self.pitch
        p.resolution, p.boundary_cells = s.grid_resolution, s.boundary_cells
        p.origin[:] = list(s.grid_origin)
        p.spacing, p.time_step = s.grid_spacing, s.time_step
        p.gravity[:] = list(s.gravity)
        p.material = 1 if self.is_ding else 0
        if self.is_ding:
            p.ding = ding_params(mc, sim.material.ding_config, s.time_step)
        else:
            p.ding.shear_modulus, p.ding.lame_lambda = mc.shear_modulus, mc.lame_lambda
        p.transport, p.gas, p.settling = int(self.transport), int(self.gas), int(settling)
        p.density = mc.density
        p.elastic_modulus = mc.lame_lambda + 2 * mc.shear_modulus
        p.cfl_limit = s.cfl_limit
        if self.transport:
            c = sim.transport.config
            p.scalar = scalar_params(c, s, settling)
            p.conductivity = 0.0 if settling else c.conductivity
            p.diffusivity = 0.0 if settling else c.water_diffusivity
            p.initial_saturation = c.initial_saturation
            p.water_stress = c.water_stress if c.water_enabled else 0.0
        if self.gas:
            d = sim.material.ding_config
            p.gas_ambient_pressure = d.gas_ambient_pressure_pa
            p.gas_peak, p.gas_width = d.gas_reaction_temperature_k, d.gas_reaction_width_k
        if self.surrogate is not None:
            p.surrogate = C.pointer(self.surrogate)
        return p

    def constants(self, settling):
        sim = self.sim
        c = BkConstants()
        c.volume = _p(sim.particle_data.reference_volumes)
        c.mass = _p(sim.particle_data.particle_masses)
        if self.transport:
            c.capacity, c.dry_mass = _p(sim.transport.capacities), _p(sim.transport.dry_masses)
            c.heat_parameter = _p(sim.transport._zero_parameter if settling else sim.transport.heat_transfer_parameter)
        if self.is_ding:
            c.viscosity_parameter = _p(sim.material.viscosity_parameter)
            rates = sim.material.production_parameter
            c.gas_rate = _p(rates)
            c.gas_rate_per_particle = int(rates.shape[0] == self.n and self.n > 1)
        return c

    def mechanics_grid(self, own_transport=False):
        """A second grid (its own node arrays and active boxes), so that recomputed substeps leave
        the simulator's grid holding its last substep. With ``own_transport`` it also has its own
        transport fields and node (dT, dW/W), which a run with keep_fields leaves in place."""
        R = self.sim.simulation_config.grid_resolution
        dev = self.sim.device
        empty = [2 ** 31 - 1] * 3 + [-2 ** 31] * 3
        fields, dTr = self.fields, self.node_dT_ratio
        if own_transport and self.transport:
            fields = [torch.zeros(R ** 3, dtype=torch.float64, device=dev) for _ in range(7)]
            dTr = torch.zeros(R ** 3, 2, dtype=torch.float64, device=dev)
        tensors = dict(node_pm=torch.zeros(R ** 3, 4, dtype=torch.float32, device=dev),
                       node_v=torch.zeros(R ** 3, 4, dtype=torch.float32, device=dev),
                       bounds=torch.tensor(empty + empty + empty, dtype=torch.int32, device=dev),
                       fields=fields, node_dT_ratio=dTr)  # kept alive with the grid
        grid = BkGrid()
        grid.node_pm, grid.node_v, grid.bounds = (_p(tensors[k]) for k in ("node_pm", "node_v", "bounds"))
        grid.node_dT_ratio = _p(dTr)
        for k in range(7):
            grid.fields[k] = _p(fields[k])
        return grid, tensors

    def batch_instance(self, state_a, state_b):
        """This simulator as one entry of a bk_batch_create table: the ping-pong pair (state_a,
        state_b), its grid, surface, flags and constants (past settling, lean diagnostics)."""
        if self.prescatter_pending:
            raise RuntimeError("transport fields are scattered ahead for a substep outside the batch")
        inst = BkBatchInstance()
        p = self.params(False)
        p.status = _p(self.status)
        inst.params = p
        for k, st in enumerate((state_a, state_b)):
            inst.states[k] = state_struct(st, self.is_ding, self.transport, self.gas)
            if self.transport:
                inst.water_losses[k] = _p(st.transport_state.water_losses)
                inst.heat_exchanges[k] = _p(st.transport_state.heat_exchanges)
        inst.constants = self.constants(False)
        inst.grid = self.grid
        inst.surface = self.surface
        inst.diagnostics.max_residuals = _p(self.max_residuals)
        inst.flags = self.flags
        return inst

    # ---------------------------------------------------------------- launch
    def prescatter_allowed(self):
        """Whether the G2P kernel may scatter the next substep's transport fields ahead (transport on,
        exact return map)."""
        sur = self.surrogate
        return bool(self.transport) and not (sur is not None and sur.packed)

    def run(self, state_in, state_out, settling, phases, full_diagnostics, grid=None, keep_fields=False,
            prescattered=False, prescatter_next=False, accumulate=None):
        """One substep through bk_substep. ``prescattered``: the previous run scattered this substep's
        transport fields ahead (its ``prescatter_next``), so the scalar P2G is skipped;
        ``prescatter_next``: scatter the next substep's, which must start from ``state_out`` with
        nothing changed in between. ``accumulate``: a transport state whose water-loss and
        heat-exchange accumulators the surface kernel advances (in place of accumulate_surface)."""
        p = self.params(settling)
        p.keep_transport_fields = int(keep_fields)
        p.transport_prescattered = int(prescattered)
        p.transport_prescatter_next = int(prescatter_next)
        p.status = _p(self.status)
        own_grid = grid is None
        if own_grid and (phases & PHASE_TRANSPORT) and self.transport:
            if prescattered and not self.prescatter_pending:
                raise RuntimeError("no transport fields were scattered ahead for this substep")
            # fields scattered ahead that this substep does not use are cleared first
            p.transport_prescatter_stale = int(self.prescatter_pending and not prescattered)
            self.prescatter_pending = False
        cst = self.constants(settling)
        sin = state_struct(state_in, self.is_ding, self.transport, self.gas)
        sout = state_struct(state_out, self.is_ding, self.transport, self.gas)
        diag = BkDiagnostics()
        diag.max_residuals = _p(self.max_residuals)
        if full_diagnostics and self.is_ding:
            m = state_out.material_state
            diag.plastic_gradients = _p(m.plastic_gradients)
            diag.return_residuals = _p(m.return_residuals)
            diag.porosity_residuals = _p(m.porosity_residuals)
        # (under a KernelTimer the library times bk_substep's kernels one by one)
        stream = _lib.stream_handle()
        sf = self.surface
        if accumulate is not None and self.transport and (phases & PHASE_TRANSPORT):
            sf.accumulate_water_losses = _p(accumulate.water_losses)
            sf.accumulate_heat_exchanges = _p(accumulate.heat_exchanges)
            sf.accumulate_time_step = self.sim.simulation_config.time_step
        try:
            rc = self.lib.bk_substep(C.byref(p), C.byref(sin), C.byref(sout), C.byref(cst),
                                     C.byref(self.grid if grid is None else grid),
                                     C.byref(sf), C.byref(diag), C.byref(self.flags), int(phases), stream)
        finally:
            sf.accumulate_water_losses = sf.accumulate_heat_exchanges = None
        if rc != 0:
            raise RuntimeError(f"bk_substep failed ({rc}): {self.lib.bk_last_error().decode(errors='replace')}")
        if own_grid and (phases & PHASE_MECHANICS):
            self.prescatter_pending = bool(prescatter_next)

    def step_summary(self, state, out=None, out_ptr=None):
        """(grid mass of the last substep, kinetic energy of ``state``) as a float64 device tensor,
        or into the 2 doubles at device address ``out_ptr``."""
        dev = self.sim.device
        if out is None and out_ptr is None:
            out = torch.empty(2, dtype=torch.float64, device=dev)
        if getattr(self, "_summary_scratch", None) is None:
            self._summary_scratch = torch.empty(2 * 296, dtype=torch.float64, device=dev)
        p = self.params(False)
        cst = self.constants(False)
        s = state_struct(state, self.is_ding, self.transport, self.gas)
        _lib.call_raw(self.lib.bk_step_summary, "bk_step_summary", C.byref(p), C.byref(s), C.byref(cst),
                      C.byref(self.grid), out.data_ptr() if out_ptr is None else out_ptr,
                      self._summary_scratch.data_ptr(), _lib.stream_handle())
        return out

    def check_state(self, state):
        """CheckState's inputs (the CHECK_SLOTS values) for ``state``, the simulator's vertex positions
        and grid, from one device reduction (bk_check_state) and one copy to the host."""
        sim = self.sim
        dev = sim.device
        if getattr(self, "_check_out", None) is None:
            self._check_out = torch.zeros(len(CHECK_SLOTS), dtype=torch.float64, device=dev)
            self._check_scratch = torch.empty(CHECK_BLOCKS * len(CHECK_SLOTS), dtype=torch.float64, device=dev)
            self._check_tets = torch.as_tensor(np.ascontiguousarray(sim.tet_mesh.tet_indices, dtype=np.int32),
                                               device=dev)
        c = BkCheckInputs()
        c.n = sim.particle_data.particle_count
        c.pitch = arrays.layout_pitch(state.deformation_gradients)
        c.x, c.v = _p(state.particle_positions), _p(state.particle_velocities)
        c.F, c.C = _p(state.deformation_gradients), _p(state.affine_velocities)
        c.reference_volume = _p(sim.particle_data.reference_volumes)
        c.mass = _p(sim.particle_data.particle_masses)
        c.sim_flags = _p(sim.error_flags)
        mc = sim.material.material_config
        c.density = mc.density
        if self.transport:
            ts = state.transport_state
            c.water, c.dry_mass, c.temperature = _p(ts.water_masses), _p(sim.transport.dry_masses), _p(ts.temperatures)
            c.transport_flags = _p(sim.transport.error_flags)
            tc = sim.transport.config
            c.water_enabled = int(tc.water_enabled)
            c.water_density, c.water_stress = tc.water_density, tc.water_stress
        if self.is_ding:
            ms = state.material_state
            c.Fe, c.ding_flags = _p(ms.elastic_gradients), _p(sim.material.error_flags)
            if not self.transport:
                c.material_temperature = _p(ms.temperatures)
            if self.gas:
                c.porosity, c.gas_moles = _p(ms.porosities), _p(ms.gas_moles)
                c.gas_modulus = mc.lame_lambda + 2.0 * mc.shear_modulus
                c.initial_porosity = sim.material.ding_config.porosity
            if sim.diagnostics == "full":
                c.return_residuals = _p(ms.return_residuals)
            c.max_residuals = _p(self.max_residuals)
        cfg = sim.simulation_config
        for a in range(3):
            c.origin[a] = cfg.grid_origin[a]
        c.spacing, c.resolution = cfg.grid_spacing, cfg.grid_resolution
        c.node_pm, c.box = _p(self.node_pm), self.bounds.data_ptr() + 6 * 4  # the last substep's box
        verts = sim.vertex_positions
        c.vertex_count, c.vertex_pitch, c.vertices = verts.shape[0], arrays.layout_pitch(verts), _p(verts)
        c.tet_count, c.tets = self._check_tets.shape[0], _p(self._check_tets)
        c.substep_status = _p(self.status)
        _lib.call_raw(self.lib.bk_check_state, "bk_check_state", C.byref(c), _p(self._check_out),
                      _p(self._check_scratch), _lib.stream_handle())
        return dict(zip(CHECK_SLOTS, self._check_out.tolist()))

    def accumulate_surface(self, transport_state):
        if not self.transport or self.surface.owner_count == 0:
            return
        _lib.call_raw(self.lib.bk_surface_accumulate, "bk_surface_accumulate", C.byref(self.surface),
                      self.sim.simulation_config.time_step, _p(transport_state.water_losses),
                      _p(transport_state.heat_exchanges), _lib.stream_handle())

    def materialize(self, state, plastic=True):
        """Fill the derivable reference fields of ``state`` from its primary arrays."""
        p = self.params(False)
        cst = self.constants(False)
        s = state_struct(state, self.is_ding, self.transport, self.gas)
        m, t = state.material_state, state.transport_state
        args = [None] * 8
        if self.is_ding:
            args[0] = _p(m.plastic_gradients) if plastic else None
            args[1] = _p(m.temperatures) if self.transport else None
            args[2] = _p(m.reference_densities)
            args[3], args[4] = _p(m.yield_stresses), _p(m.viscosities)
            args[5] = _p(m.gas_pressures) if self.gas else None
        if self.transport:
            args[6], args[7] = _p(t.saturations), _p(t.particle_masses)
        _lib.call_raw(self.lib.bk_materialize, "bk_materialize", C.byref(p), C.byref(s), C.byref(cst), *args,
                      _lib.stream_handle())
