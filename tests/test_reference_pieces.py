"""The engine and the oracle against the reference's own code, for the two
pieces of the matvec path that compile from the reference's sources alone
(oracle/_ref, built by oracle/Makefile from the reference tree):

* the scaled modified spherical Bessel functions: the reference forms
  b[n] = sqrt(pi / 2x) I_{n+1/2}(x) / scal^n from Cody's RIBESL
  (src/fmm/fmm_math_funcs.h:24-113, src/fmm/bessel_gamma.h:269); the
  engine's host tables and the oracle use Miller's backward recurrence;
* the 1512-entry interaction list (src/fmm/interaction_list.h:93-1607),
  which the engine and the oracle generate from its rule instead of storing.

Skipped when oracle/_ref is not built (the reference tree is absent)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import native
import oracle as O

ROOT = Path(__file__).resolve().parent.parent
REF = O.ref_lib()
pytestmark = pytest.mark.skipif(REF is None, reason="oracle/_ref not built (no reference tree)")


@pytest.fixture(scope="module")
def shim():
    L = native.load("special_functions_shim", [ROOT / "beep3_b200" / "csrc" / "fmm_tables.cpp",
                                                ROOT / "beep3_b200" / "csrc" / "fmm_tables.h",
                                                ROOT / "oracle" / "fmm_oracle.cpp"])
    d, i, p = C.c_double, C.c_int, C.c_void_p
    L.shim_engine_bessel_in.argtypes = [d, d, i, p]
    L.shim_oracle_i_n.argtypes = [d, d, i, p]
    L.shim_engine_interaction_list.argtypes = [p]
    L.shim_engine_interaction_list.restype = i
    return L


def reference_i_n(scal, x, nb):
    """fmm::i_n restated around the reference's compiled RIBESL: unscaled
    (ize = 1) I_{n+1/2}(x), times sqrt(pi/2x) / scal^n, the scale factor set
    to zero once a value falls to 1e-300 or below."""
    b = np.zeros(nb + 2)
    REF.ref_ribesl(x, 0.5, nb + 1, 1, b.ctypes.data)
    out = np.zeros(nb + 1)
    const = np.sqrt(np.pi / 2 / x)
    for i in range(nb + 1):
        out[i] = b[i] * const
        const /= scal
        if abs(out[i]) <= 1e-300:
            const = 0.0
    return out


@pytest.mark.parametrize("fn", ["shim_engine_bessel_in", "shim_oracle_i_n"])
def test_i_n_matches_the_reference_ribesl(shim, fn):
    rng = np.random.default_rng(7)
    # arguments the FMM tables use: beta * r up to the cube size at kappa <= 0.15
    xs = np.concatenate([[1.5e-4, 1e-3, 0.05, 0.3, 1.0, 4.0, 17.0, 60.0, 99.0], 10.0 ** rng.uniform(-3.5, 2.0, 60)])
    worst = 0.0
    for nb in (9, 12, 18):
        for x in xs:
            for scal in (1.0, 0.3, 0.05):
                ref = reference_i_n(scal, float(x), nb)
                b = np.zeros(nb + 1)
                getattr(shim, fn)(scal, float(x), nb, b.ctypes.data)
                keep = np.abs(ref) > 1e-280
                worst = max(worst, float(np.max(np.abs(b[keep] - ref[keep]) / np.abs(ref[keep]))))
    assert worst < 1e-13, worst


def entries(fn) -> set:
    n = fn(None)
    a = np.zeros((n, 7), np.int32)
    assert fn(a.ctypes.data) == n
    return n, {tuple(int(v) for v in r) for r in a}


def test_interaction_lists_equal_the_reference_table(shim):
    n_ref, ref = entries(REF.ref_interaction_list)
    assert n_ref == 1512 and len(ref) == 1512
    n_or, orc = entries(O.lib().or_interaction_list)
    assert n_or == 1512 and orc == ref
    # the engine numbers children 0..7 where the reference uses 1..8
    n_en, eng = entries(shim.shim_engine_interaction_list)
    assert n_en == 1512
    assert {(nb, d, t + 1, s + 1, dx, dy, dz) for nb, d, t, s, dx, dy, dz in eng} == ref
