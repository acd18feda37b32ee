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


def test_batch_entry_points_validate_arguments():
    """bp_problem_create_batch and bp_solve_batch reject bad arguments before
    any device work (no GPU needed)."""
    L = N.lib()
    h = C.c_void_p()
    prm = N.bp_params(0.1, 1e-10, (C.c_double * 3)(0, 0, 0), 50.0, 100, 9, N.BP_PREC_MIXED, 0)
    centres = np.zeros(6)
    insts = (N.bp_instance * 2)()
    bad_first = np.array([0, 2, 2], np.int32)  # the second scenario has no instance
    assert L.bp_problem_create_batch(None, insts, 2, N.ptr(bad_first), 2, N.ptr(centres), C.byref(prm),
                                     C.byref(h)) == N.BP_ERR_INVALID
    assert b"every scenario needs an instance" in L.bp_last_error()
    short = np.array([0, 1, 1], np.int32)  # does not end at n_instances
    assert L.bp_problem_create_batch(None, insts, 3, N.ptr(short), 2, N.ptr(centres), C.byref(prm),
                                     C.byref(h)) == N.BP_ERR_INVALID
    assert b"scenario_first" in L.bp_last_error()
    nan_centres = np.array([0.0, np.nan, 0.0, 0.0, 0.0, 0.0])
    ok_first = np.array([0, 1, 2], np.int32)
    assert L.bp_problem_create_batch(None, insts, 2, N.ptr(ok_first), 2, N.ptr(nan_centres), C.byref(prm),
                                     C.byref(h)) == N.BP_ERR_INVALID
    assert L.bp_problem_create_batch(None, insts, 2, N.ptr(ok_first), 2, N.ptr(centres), C.byref(prm),
                                     C.byref(h)) == N.BP_ERR_INVALID  # no context
    rhs = np.zeros(4)
    x = np.zeros(4)
    assert L.bp_solve_batch(None, N.ptr(rhs), N.ptr(x), 1e-6, 10, 0, None, None) == N.BP_ERR_INVALID
    its = np.zeros(2, np.int32)
    rr = np.zeros(2)
    assert L.bp_solve_batch(None, N.ptr(rhs), N.ptr(x), 1e-6, 10, 0, N.ptr(its), N.ptr(rr)) == N.BP_ERR_INVALID


def test_header_constants_match_the_binding():
    """Every enum constant of the C header (status codes, precisions, flags)
    has the same value in the Python binding."""
    h = (Path(__file__).resolve().parents[1] / "include" / "beep3_b200.h").read_text()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    consts = dict((k, int(v)) for k, v in re.findall(r"\b(BP_[A-Z0-9_]+)\s*=\s*(\d+)", h))
    assert {"BP_OK", "BP_ERR_NOT_CONVERGED", "BP_PREC_MIXED", "BP_FLAG_MESH_PAIR_CACHE"} <= set(consts)
    for k, v in consts.items():
        assert getattr(N, k) == v, k
