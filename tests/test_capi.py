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
