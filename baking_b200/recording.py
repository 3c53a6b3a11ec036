"""Per-step measurements of a run, buffered in memory (experiments/recording.py:38-229).

``SimulationRecorder`` keeps the reference recorder's API and measurement keys: attach it as
``simulator.result_recorder`` and ``Step()`` records after every substep. ``Measure()`` is one
device reduction (``bk_measure_state``: particle volume, porosity, gas, temperature, water, energy
and saturation statistics, mesh extents, tet volumes and inversions) and one read of its
BK_MEASURE_SLOTS doubles, where the reference pulls every state array to the host each substep.
``Finish()`` writes the run folder's data files (summary.json, the history CSVs, the final state
and surface, queued snapshots); the SVG plots are left out.
"""

from __future__ import annotations

import csv
import ctypes as C
import json
from dataclasses import asdict
from datetime import datetime, timezone
from pathlib import Path
from uuid import uuid4

import numpy as np
import torch

from . import _lib, arrays
from .physics.materials.ding import DingMaterial

P = C.c_void_p


class BkMeasureInputs(C.Structure):
    _fields_ = [("n", C.c_int64), ("pitch", C.c_int64), ("F", P), ("reference_volume", P),
                ("material_temperature", P), ("porosity", P), ("gelled", P), ("gas_moles", P), ("gas_pressure", P),
                ("temperature", P), ("water", P), ("saturation", P), ("water_losses", P), ("heat_exchanges", P),
                ("capacity", P), ("regions", P), ("vertex_count", C.c_int64), ("vertex_pitch", C.c_int64),
                ("vertices", P), ("tet_count", C.c_int64), ("tets", P)]


# Slots of bk_measure_state (include/baking_b200.h, BK_MEASURE_*).
SLOTS = ("particle_volume", "invalid_particles", "nonfinite", "material_t_sum", "porosity_sum", "porosity_min",
         "porosity_max", "gelled", "gas_total", "pressure_sum", "pressure_min", "pressure_max", "pore_volume",
         "t_min", "t_max", "energy", "capacity", "surface_t_sum", "surface_count", "core_t_sum", "core_count",
         "water", "water_lost", "heat_exchange", "saturation_sum", "saturation_min", "saturation_max",
         "x_min", "y_min", "z_min", "x_max", "y_max", "z_max", "mesh_volume", "inverted_tets")
MEASURE_BLOCKS = 296


def ExtractSurface(vertex_positions, tet_indices):
    """Boundary faces of a tet mesh, oriented outward, with their vertices renumbered
    (experiments/recording.py:12-35)."""
    tets = np.asarray(tet_indices)
    faces = np.concatenate([tets[:, [k for k in range(4) if k != o]] for o in range(4)])
    opposite = np.concatenate([tets[:, o] for o in range(4)])
    _, inverse, counts = np.unique(np.sort(faces, axis=1), axis=0, return_inverse=True, return_counts=True)
    if np.any(counts > 2):
        raise ValueError("Nonmanifold tet mesh: more than two cells share a face")
    boundary = counts[inverse.reshape(-1)] == 1
    surface = faces[boundary].copy()
    corners = vertex_positions[surface]
    inward = vertex_positions[opposite[boundary]] - corners[:, 0]
    normals = np.cross(corners[:, 1] - corners[:, 0], corners[:, 2] - corners[:, 0])
    flip = np.einsum("ij,ij->i", normals, inward) > 0
    surface[flip, 1], surface[flip, 2] = surface[flip, 2].copy(), surface[flip, 1].copy()
    used, remapped = np.unique(surface, return_inverse=True)
    return vertex_positions[used].copy(), remapped.reshape(-1, 3)


class SimulationRecorder:
    def __init__(self, simulator, experiment_config):
        self.simulator = simulator
        self.experiment_config = experiment_config
        self.pending_snapshots = []
        self.finished_path = None
        self._prepare()
        self.Reset()

    # ------------------------------------------------------------ device set-up
    def _prepare(self):
        sim = self.simulator
        dev = sim.device
        self._lib = _lib.load()
        self._out = torch.zeros(len(SLOTS), dtype=torch.float64, device=dev)
        self._scratch = torch.empty(MEASURE_BLOCKS * len(SLOTS), dtype=torch.float64, device=dev)
        self._tets = torch.as_tensor(np.ascontiguousarray(sim.tet_mesh.tet_indices, dtype=np.int32), device=dev)
        self._regions = None
        if sim.transport is not None:
            self._regions = self._particle_regions()
            config = sim.transport.config
            volumes = np.asarray(sim.particle_samples.reference_volumes, dtype=np.float64)
            self._initial_water = config.water_density * config.initial_saturation * volumes.sum()

    def _particle_regions(self):
        """Per-particle region bits in the simulator's current particle order: bit 0, owns a
        boundary face; bit 1, the initial core, radius < 0.4 of the largest distance of a sampled
        position from the mesh centroid (recording.py:80-86)."""
        sim = self.simulator
        self._sort_count = sim.sort_count
        regions = np.zeros(sim.particle_data.particle_count, dtype=np.uint8)
        regions[sim.transport.owners.cpu().numpy()] |= 1
        positions = np.asarray(sim.particle_samples.particle_positions)
        center = np.mean(sim.tet_mesh.vertex_positions, axis=0)
        radius = np.linalg.norm(positions - center, axis=1)
        core = radius < 0.4 * radius.max()
        if not core.any():
            core = radius == radius.min()
        regions[core] |= 2
        return torch.as_tensor(regions, device=sim.device)

    def _inputs(self, state):
        sim = self.simulator
        if self._regions is not None and sim.sort_count != self._sort_count:
            self._regions = self._particle_regions()  # the particles were reordered
        m = BkMeasureInputs()
        m.n = sim.particle_data.particle_count
        m.pitch = arrays.layout_pitch(state.deformation_gradients)
        m.F = state.deformation_gradients.data_ptr()
        m.reference_volume = sim.particle_data.reference_volumes.data_ptr()
        if isinstance(sim.material, DingMaterial):
            ms = state.material_state
            m.material_temperature, m.porosity = ms.temperatures.data_ptr(), ms.porosities.data_ptr()
            m.gelled = ms.gelled.data_ptr()
            if sim.material.ding_config.gas_enabled:
                m.gas_moles, m.gas_pressure = ms.gas_moles.data_ptr(), ms.gas_pressures.data_ptr()
        if state.transport_state is not None:
            t = state.transport_state
            m.temperature, m.water, m.saturation = t.temperatures.data_ptr(), t.water_masses.data_ptr(), \
                t.saturations.data_ptr()
            m.water_losses, m.heat_exchanges = t.water_losses.data_ptr(), t.heat_exchanges.data_ptr()
            m.capacity = sim.transport.capacities.data_ptr()
            m.regions = self._regions.data_ptr()
        verts = sim.vertex_positions
        m.vertex_count, m.vertex_pitch = verts.shape[0], arrays.layout_pitch(verts)
        m.vertices = verts.data_ptr()
        m.tet_count, m.tets = self._tets.shape[0], self._tets.data_ptr()
        return m

    def _reduce(self):
        """The measurement slots of the current state, and the first yield stress and viscosity."""
        sim = self.simulator
        sim.UpdateMesh()
        state = sim.current_state
        m = self._inputs(state)
        _lib.call_raw(self._lib.bk_measure_state, "bk_measure_state", C.byref(m), self._out.data_ptr(),
                      self._scratch.data_ptr(), _lib.stream_handle())
        parts = [self._out]
        if isinstance(sim.material, DingMaterial):
            ms = state.material_state
            parts += [ms.yield_stresses[:1].double(), ms.viscosities[:1].double()]
        values = torch.cat(parts).tolist()
        return dict(zip(SLOTS, values[:len(SLOTS)])), values[len(SLOTS):]

    # -------------------------------------------------------------- measuring
    def Measure(self):
        sim = self.simulator
        r, first = self._reduce()
        if r["nonfinite"] > 0:
            raise ValueError("Cannot record nonfinite simulation state")
        n = sim.particle_data.particle_count
        values = {}
        if isinstance(sim.material, DingMaterial):
            values.update(
                temperature_k=r["material_t_sum"] / n, porosity_min=r["porosity_min"],
                porosity_mean=r["porosity_sum"] / n, porosity_max=r["porosity_max"],
                yield_stress_pa=first[0], viscosity_pa3_s=first[1], gelled_fraction=r["gelled"] / n)
            if sim.material.ding_config.gas_enabled:
                values.update(
                    gas_total_mol=r["gas_total"], gas_pressure_min_pa=r["pressure_min"],
                    gas_pressure_max_pa=r["pressure_max"], gas_pressure_mean_pa=r["pressure_sum"] / n,
                    pore_volume_m3=r["pore_volume"])
        if sim.transport is not None:
            config = sim.transport.config
            initial_energy = config.initial_temperature_k * r["capacity"]
            surface = r["surface_t_sum"] / r["surface_count"] if r["surface_count"] else float("nan")
            values.update(
                temperature_min_k=r["t_min"], temperature_max_k=r["t_max"],
                temperature_mean_k=r["energy"] / r["capacity"], temperature_surface_k=surface,
                temperature_core_k=r["core_t_sum"] / r["core_count"],
                water_mass_kg=r["water"], water_lost_kg=r["water_lost"],
                water_balance_error_kg=r["water"] + r["water_lost"] - self._initial_water,
                saturation_min=r["saturation_min"], saturation_max=r["saturation_max"],
                saturation_mean=r["saturation_sum"] / n, thermal_energy_j=r["energy"],
                heat_exchange_j=r["heat_exchange"],
                energy_balance_error_j=r["energy"] - initial_energy - r["heat_exchange"])
        return dict(**values, baking_time_s=sim.baking_time, phase="settling" if sim.IsSettling else "baking",
                    step=sim.step_count, time_s=sim.step_count * sim.simulation_config.time_step,
                    length_x_m=r["x_max"] - r["x_min"], width_z_m=r["z_max"] - r["z_min"],
                    height_y_m=r["y_max"] - r["y_min"], particle_volume_m3=r["particle_volume"],
                    mesh_volume_m3=r["mesh_volume"], inverted_tets=int(r["inverted_tets"]),
                    invalid_particles=int(r["invalid_particles"]))

    def Reset(self):
        self.settled_measurement = None
        self.expansion_history = []
        self.height_history = []
        self.pending_snapshots = []
        self.initial_measurement = self.Measure()
        self.last_measurement = self.initial_measurement
        self.height_history.append((self.initial_measurement["time_s"], self.initial_measurement["height_y_m"]))
        self.recorded_step = self.simulator.step_count
        self.expansion_history.append(dict(self.last_measurement))
        if self.experiment_config.run.snapshot_interval:
            self.QueueSnapshot()

    def Record(self):
        if self.recorded_step == self.simulator.step_count:
            return
        self.last_measurement = self.Measure()
        self.height_history.append((self.last_measurement["time_s"], self.last_measurement["height_y_m"]))
        self.recorded_step = self.simulator.step_count
        self.expansion_history.append(dict(self.last_measurement))
        interval = self.experiment_config.run.snapshot_interval
        if interval and self.simulator.step_count % interval == 0:
            self.QueueSnapshot()

    def QueueSnapshot(self):
        self.pending_snapshots.append((self.simulator.step_count, self.simulator.CaptureSnapshot()))

    # -------------------------------------------------------------- writing
    def Finish(self, status="completed", error_message="", console_text=""):
        """Write the run folder under ``run.log_path`` once and return its path
        (experiments/recording.py:140-222, without the SVG plots)."""
        if self.finished_path is not None:
            return self.finished_path
        try:
            self.Record()
        except (ValueError, RuntimeError) as record_error:
            status = "failed"
            error_message = (error_message + "; " + str(record_error)).strip("; ")
        sim = self.simulator
        run_name = datetime.now(timezone.utc).strftime("%Y%m%dT%H%M%S_%fZ") + "_" + uuid4().hex[:8]
        run_path = Path(self.experiment_config.run.log_path).expanduser() / run_name
        run_path.mkdir(parents=True, exist_ok=False)
        final = self.last_measurement
        settling_steps = sim.settling_steps if not sim.IsSettling else sim.step_count
        summary = dict(
            status=status, error=error_message,
            units=dict(length="m", volume="m^3", time="s", mass="kg", stress="Pa", temperature="K", porosity="1",
                       ding_viscosity="Pa^3 s", gas_content="mol/m^3 of reference volume", gas_amount="mol"),
            initial=self.initial_measurement, settled=self.settled_measurement, final=final,
            settling_steps=settling_steps, settling_reason=sim.settling_reason,
            settling_diagnostics=sim.settling_diagnostics,
            actual_settling_duration_s=settling_steps * sim.simulation_config.time_step,
            attempted_step=sim.step_count, parameters=asdict(self.experiment_config), actual_device=sim.device_name,
            sample_count=len(self.height_history), total_mass_kg=float(sim.Masses().double().sum()))
        if final["step"] == sim.step_count:
            vertices, faces = ExtractSurface(arrays.to_numpy(sim.vertex_positions), sim.tet_mesh.tet_indices)
            with (run_path / "final_surface.obj").open("w", encoding="ascii") as f:
                f.write("# Units: metres. Boundary of the reconstructed tetrahedral mesh.\n")
                for v in vertices:
                    f.write("v " + " ".join(format(float(x), ".9g") for x in v) + "\n")
                for face in faces:
                    f.write("f " + " ".join(str(int(k) + 1) for k in face) + "\n")
            sim.SaveSnapshot(run_path / "final_state.npz")
        else:
            summary["surface_omitted"] = "Final state invalid; measurements refer to last valid recorded state"
        with (run_path / "height_history.csv").open("w", newline="", encoding="ascii") as f:
            w = csv.writer(f)
            w.writerow(["time_s", "height_y_m"])
            w.writerows(self.height_history)
        if sim.transport is not None:
            thermal = ["time_s", "baking_time_s", "phase"] + [k for k in self.expansion_history[0] if k.startswith(
                ("temperature_", "water_", "saturation_", "thermal_", "heat_", "energy_"))]
            self._write_csv(run_path / "thermal_water_history.csv", thermal)
        self._write_csv(run_path / "expansion_history.csv", list(self.expansion_history[0]))
        if isinstance(sim.material, DingMaterial):
            names = ["time_s", "temperature_k", "porosity_min", "porosity_mean", "porosity_max", "yield_stress_pa",
                     "viscosity_pa3_s", "gelled_fraction"]
            if sim.material.ding_config.gas_enabled:
                names += ["gas_total_mol", "gas_pressure_min_pa", "gas_pressure_max_pa", "gas_pressure_mean_pa",
                          "pore_volume_m3"]
            self._write_csv(run_path / "material_history.csv", names)
        for step, data in self.pending_snapshots:
            np.savez_compressed(run_path / f"snapshot_{step:07d}.npz", **data)
        (run_path / "summary.json").write_text(json.dumps(summary, indent=2, ensure_ascii=True, allow_nan=False),
                                               encoding="utf-8")
        (run_path / "console.log").write_text(console_text, encoding="utf-8")
        self.finished_path = run_path
        return run_path

    def _write_csv(self, path, names):
        with path.open("w", newline="", encoding="ascii") as f:
            w = csv.DictWriter(f, fieldnames=names, extrasaction="ignore")
            w.writeheader()
            w.writerows(self.expansion_history)
