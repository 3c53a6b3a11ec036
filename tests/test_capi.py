"""The C-ABI library loads without a GPU, exports every entry point include/baking_b200.h
declares, and every ctypes binding has the declared number of arguments."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "baking_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for match in re.finditer(r"BK_API\s+[\w\s\*]+?\b(bk_\w+)\s*\(([^)]*)\)\s*;", text):
        args = match.group(2).strip()
        out[match.group(1)] = 0 if args in ("", "void") else len(args.split(","))
    return out


def test_header_declares_entry_points():
    funcs = declared_functions()
    assert "bk_substep" in funcs and "bk_update_ding" in funcs and "bk_diffuse_grid" in funcs
    assert len(funcs) >= 20


def test_library_exports_every_declared_symbol():
    from baking_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} missing from {lib_path.name}"


def test_bindings_match_declared_arity():
    from baking_b200 import _lib
    from baking_b200 import surrogate
    from baking_b200.physics import adjoint, substep
    funcs = declared_functions()
    bindings = dict(_lib.SIGNATURES)
    bindings.update(substep._SIGS)
    bindings.update(surrogate.SIGNATURES)
    bindings.update(adjoint._SIGNATURES)
    for name, argtypes in bindings.items():
        assert name in funcs, f"{name} bound but not declared"
        assert len(argtypes) == funcs[name], f"{name}: {len(argtypes)} bound vs {funcs[name]} declared"


def test_oracle_library_builds_and_exports():
    from oracle import ora
    lib = ora.lib()
    for name in ("ora_particle_to_grid", "ora_update_ding", "ora_diffuse_grid", "ora_svd3"):
        assert hasattr(lib, name)


def test_permute_particles_rejects_bad_arguments_before_any_device_work():
    """Argument checks of bk_permute_particles run on the host before any CUDA call, so they are
    exercised here without a GPU: n beyond the int32 order, scratch not 256-byte aligned and an
    array not aligned to its element size each return BK_ERR_ARGUMENT with a message."""
    from baking_b200 import _lib
    lib = _lib.load()
    fn = lib.bk_permute_particles  # bound by _lib.load() with the header's argument types

    class Arr(ctypes.Structure):
        _fields_ = [("data", ctypes.c_void_p), ("pitch", ctypes.c_int64), ("planes", ctypes.c_int32),
                    ("element_bytes", ctypes.c_int32)]

    table = (Arr * 1)()
    table[0].data, table[0].pitch, table[0].planes, table[0].element_bytes = 4096, 1 << 20, 1, 8
    aligned = 1 << 20
    cases = [
        ((2 ** 31, 256, 1, ctypes.addressof(table), aligned, 1 << 40, None), "int32"),
        ((1000, 256, 1, ctypes.addressof(table), aligned + 8, 1 << 40, None), "256-byte"),
    ]
    for args, message in cases:
        assert fn(*args) != 0
        assert message in lib.bk_last_error().decode()
    table[0].data = 4096 + 4
    assert fn(1000, 256, 1, ctypes.addressof(table), aligned, 1 << 40, None) != 0
    assert "element size" in lib.bk_last_error().decode()


def test_batch_entry_points_reject_bad_arguments_without_a_gpu():
    """bk_batch_create refuses a null or empty table and bk_batch_substep a null batch or a parity
    other than 0 and 1, before any CUDA call; destroying a null batch is a no-op."""
    from baking_b200.physics import substep
    lib = substep._declare()
    handle = ctypes.c_void_p()
    assert lib.bk_batch_create(None, 0, ctypes.byref(handle)) != 0
    assert "empty batch" in lib.bk_last_error().decode()
    table = (substep.BkBatchInstance * 1)()
    assert lib.bk_batch_create(table, 0, ctypes.byref(handle)) != 0
    assert lib.bk_batch_substep(None, 0, 3, 0, 0, None) != 0
    assert "parity" in lib.bk_last_error().decode()
    assert lib.bk_batch_destroy(None) == 0
