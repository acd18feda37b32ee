"""The C ABI library loads and exports every entry point its header declares;
host-only entry points validate their arguments (no device needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent


def declared_functions() -> list[str]:
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(bp_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_symbols_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = C.CDLL(str(N.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers every declared entry point
    assert set(names) <= set(N.exported_symbols()), set(names) - set(N.exported_symbols())


def test_abi_version_and_errors():
    L = N.lib()
    assert L.bp_abi_version() == 1
    h = C.c_void_p()
    assert L.bp_geom_create(0, None, None, 0, None, 0, 4, 0, C.byref(h)) == N.BP_ERR_INVALID
    assert b"bad arguments" in L.bp_last_error()
    assert L.bp_tree_create(0, None, None, 1.0, 10, C.byref(h)) == N.BP_ERR_INVALID
    assert L.bp_problem_info_get(None, None) == N.BP_ERR_INVALID


def test_tree_rejects_points_outside_cube():
    from beep3_b200.beep import build_tree
    pts = np.array([[0.0, 0.0, 0.0], [5.0, 0.0, 0.0]])
    with pytest.raises(b.BeepError):
        build_tree(pts, np.zeros(3), 2.0, 10)


def test_energy_entry_point_validates():
    L = N.lib()
    e = C.c_double()
    assert L.bp_energy(None, 0, 1, None, None, 40.0, None, C.byref(e)) == N.BP_ERR_INVALID


def test_posed_rhs_entry_point_validates():
    L = N.lib()
    rhs = np.zeros(2)
    counts = (C.c_int32 * 1)(0)
    ptrs = (C.c_void_p * 1)(None)
    assert L.bp_rhs_posed(None, C.cast(ptrs, C.c_void_p), C.cast(counts, C.c_void_p), 80.0,
                          N.ptr(rhs)) == N.BP_ERR_INVALID
    assert b"bad argument" in L.bp_last_error()
