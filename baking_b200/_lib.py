"""Loader for the sm_100a library ``libbaking_b200.so`` (ctypes over the C ABI).

The product path has no CPU fallback: if the library or a CUDA device is
missing, the first call raises.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import torch

PACKAGE = Path(__file__).resolve().parent
LIBRARY = PACKAGE / "libbaking_b200.so"

P = C.c_void_p
I32, I64, F32, F64 = C.c_int32, C.c_int64, C.c_float, C.c_double


class BkDingParams(C.Structure):
    _fields_ = [("coupled_porosity", C.c_int32), ("temperature_enabled", C.c_int32), ("shear_modulus", C.c_float),
                ("lame_lambda", C.c_float), ("yield_stress", C.c_float), ("initial_porosity", C.c_float),
                ("time_step", C.c_float), ("temperature_knots", C.c_float * 4), ("yield_factors", C.c_float * 4),
                ("viscosity_factors", C.c_float * 4)]


class BkScalarParams(C.Structure):
    _fields_ = [("oven_temperature", C.c_float), ("tray_temperature", C.c_float), ("tray_transfer", C.c_float),
                ("surface_loss", C.c_float), ("water_density", C.c_float), ("latent_heat", C.c_float),
                ("water_enabled", C.c_int32), ("origin", C.c_float * 3), ("spacing", C.c_float),
                ("resolution", C.c_int32)]


# name -> argtypes (an int status unless RESTYPES says otherwise; bk_version and bk_last_error are bound apart)
SIGNATURES = {
    "bk_particle_to_grid": [I64, I64, P, P, P, P, P, P, P, P, F32, I32, F32, P, P],
    "bk_update_grid": [I32, P, P, I32, P, F32, P],
    "bk_grid_to_particle": [I64, I64, P, P, P, P, P, P, P, P, F32, I32, F32, P, P],
    "bk_compute_elastic_stress": [I64, I64, P, P, F32, F32, P, P],
    "bk_update_ding": [I64, I64] + [P] * 18 + [P, P],
    "bk_combine_gas_stress": [I64, I64, P, P, P, P, P, P, P, F32, F32, P, F32, F32, F32, F32, P],
    "bk_refresh_gas": [I64, I64, P, P, P, P, P, P, P],
    "bk_reconstruct_mesh_vertices": [I64, I64, P, P, I64, P, P, P, P, I64, P, P, P],
    "bk_surface_areas": [I64, I64, P, P, P, P, P, F32, F32, P],
    "bk_scalar_to_grid": [I64, I64] + [P] * 9 + [P, P, P, P, P, P],
    "bk_grid_fields": [I64, P, P, P, P, P, P, F32, P],
    "bk_diffuse_grid": [I64] + [P] * 11 + [F32, F32, F32, I32, F32, I32, F32, P],
    "bk_scalar_to_particles": [I64, I64] + [P] * 21 + [F32, P, F32, I32, F32, P, P],
    "bk_local_gas": [I64, I64, P, P, P, P, P, P, P, P, I32, F32, F32, F32, F32, I32, P],
    "bk_water_stress": [I64, I64, P, P, P, P, F32, F32, P],
    "bk_saturations": [I64, I64, P, P, P, P, F32, P],
    "bk_settling_metrics": [I64, I64, P, P, P, P, P, F32, P],
    "bk_measure_state": [P, P, P, P],
    "bk_step_summary": [P, P, P, P, P, P, P],
    "bk_solve_porosity": [I64, P, P, P, P, P, P, F32, P, P, P],
    "bk_porosity_coefficient": [I64, P, P, P],
    "bk_profile_start": [],
    "bk_profile_stop": [],
    "bk_profile_select": [C.c_char_p],
    "bk_profile_report": [I32, P, I32, P, P, P],
    "bk_sort_by_cell": [I64, I64, P, P, F32, I32, P, P, I64, P],
    "bk_sort_by_cell_scratch_bytes": [I64, I32],
    "bk_permute_particles": [I64, P, I32, P, P, I64, P],
}


class BkParticleArray(C.Structure):
    _fields_ = [("data", C.c_void_p), ("pitch", C.c_int64), ("planes", C.c_int32), ("element_bytes", C.c_int32)]
# entry points whose return value is a count, not a status
RESTYPES = {"bk_sort_by_cell_scratch_bytes": C.c_int64}

_lib = None


def library_path():
    return LIBRARY


def load():
    """Load (building first if sources changed and nvcc exists) the CUDA library."""
    global _lib
    if _lib is not None:
        return _lib
    override = os.environ.get("BAKING_B200_LIBRARY")
    if override:
        # An alternative build of the same sources (for example one compiled with other flags).
        return _bind(C.CDLL(override))
    from . import build as _build
    try:
        if _build.needs_build():
            _build.build()
    except RuntimeError:
        if not LIBRARY.exists():
            raise
    if not LIBRARY.exists():
        raise RuntimeError(f"{LIBRARY} is missing; run `python -m baking_b200.build` (needs nvcc)")
    return _bind(C.CDLL(str(LIBRARY)))


def _bind(lib):
    global _lib
    lib.bk_version.restype = C.c_int
    lib.bk_version.argtypes = []
    lib.bk_last_error.restype = C.c_char_p
    lib.bk_last_error.argtypes = []
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = RESTYPES.get(name, C.c_int)
        fn.argtypes = argtypes
    _lib = lib
    return lib


def require_cuda(device=None):
    if not torch.cuda.is_available():
        raise RuntimeError("baking_b200 runs on a CUDA device (B200, sm_100a); none is available")
    return torch.device(device if device not in (None, "auto", "cuda") else "cuda:0")


class KernelTimer:
    """Per-kernel CUDA-event timing while active: the library's own events around every launch
    inside the fused entry points, plus host-side events around each other C-ABI call. ``only``
    restricts the events to one kernel name (every event pair costs the stream a few microseconds)."""

    active = None

    def __init__(self, only=None):
        self.only = only
        self.events = {}

    def __enter__(self):
        self.events = {}
        lib = load()
        lib.bk_profile_start()
        lib.bk_profile_select(self.only.encode() if self.only else None)
        KernelTimer.active = self
        return self

    def __exit__(self, *exc):
        KernelTimer.active = None
        lib = load()
        lib.bk_profile_stop()
        lib.bk_profile_select(None)

    def wants(self, name):
        return self.only is None or name == self.only

    def add(self, name, start, end):
        if name.startswith("bk_substep"):
            return  # timed kernel by kernel inside the library
        self.events.setdefault(name, []).append((start, end))

    def summary(self):
        torch.cuda.synchronize()
        out = {}
        for name, pairs in self.events.items():
            times = [a.elapsed_time(b) / 1e3 for a, b in pairs]
            out[name] = {"count": len(times), "total_s": sum(times), "mean_s": sum(times) / len(times)}
        lib = load()
        cap, kmax = 64, 64
        names = C.create_string_buffer(cap * kmax)
        totals = (C.c_double * kmax)()
        counts = (C.c_int32 * kmax)()
        got = C.c_int32(0)
        if lib.bk_profile_report(kmax, names, cap, totals, counts, C.byref(got)) != 0:
            raise RuntimeError(lib.bk_last_error().decode(errors="replace"))
        for k in range(got.value):
            name = names.raw[k * cap:(k + 1) * cap].split(b"\0", 1)[0].decode()
            if counts[k]:
                out[name] = {"count": int(counts[k]), "total_s": totals[k] / 1e3, "mean_s": totals[k] / 1e3 / counts[k]}
        return out


def call(name, *args):
    """Call one C-ABI entry point; raise RuntimeError on a nonzero status."""
    lib = load()
    timer = KernelTimer.active
    if timer is not None and timer.wants(name):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        rc = getattr(lib, name)(*args)
        end.record()
        timer.add(name, start, end)
    else:
        rc = getattr(lib, name)(*args)
    if rc != 0:
        message = lib.bk_last_error().decode(errors="replace")
        raise RuntimeError(f"{name} failed ({rc}): {message}")


def call_raw(fn, name, *args):
    """Call an already-declared C-ABI function object (timed like ``call``); raise on failure."""
    timer = KernelTimer.active
    if timer is not None and timer.wants(name):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        rc = fn(*args)
        end.record()
        timer.add(name, start, end)
    else:
        rc = fn(*args)
    if rc != 0:
        raise RuntimeError(f"{name} failed ({rc}): {load().bk_last_error().decode(errors='replace')}")


def stream_handle(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def ctypes_ref(structure):
    """Address of a ctypes parameter struct, for a `const Bk*Params*` argument."""
    return C.addressof(structure)
