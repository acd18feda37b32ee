"""The FMM's special functions against scipy, an implementation neither the
engine nor the oracle shares code with.

The reference computes the scaled modified spherical Bessel functions as
b[n] = sqrt(pi / 2x) I_{n+1/2}(x) / scal^n with Cody's RIBESL, the series
1 + x^2 / (2(2n+3)) for x <= 1e-4 and zero above x = 100
(src/fmm/fmm_math_funcs.h:24-113); the associated Legendre functions with
the Condon-Shortley phase for |x| <= 1 (lgndr, :115-141) and scaled as
scal^n P_n^m(x) without it for x > 1 (lgndrgt1, :143-207).  The engine's
host tables (beep3_b200/csrc/fmm_tables.cpp) and the oracle replace RIBESL
with Miller's backward recurrence; both are checked here.  The device copies
of the same recurrences (bessel_in_dev, legendre_dev in fmm.cu) tabulate the
P2M and L2P bases, whose FMM results the GPU tests hold to the oracle's at
1e-8, so they are pinned through those tests.
"""
import ctypes as C
from math import factorial

import numpy as np
import pytest
from numpy.polynomial import legendre as npleg
from scipy import special

import native



@pytest.fixture(scope="module")
def shim():
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    L = native.load("special_functions_shim", [root / "beep3_b200" / "csrc" / "fmm_tables.cpp",
                                                root / "beep3_b200" / "csrc" / "fmm_tables.h",
                                                root / "oracle" / "fmm_oracle.cpp"])
    d, i, p = C.c_double, C.c_int, C.c_void_p
    L.shim_engine_bessel_in.argtypes = [d, d, i, p]
    L.shim_oracle_i_n.argtypes = [d, d, i, p]
    L.shim_engine_legendre_gt1.argtypes = [i, d, d, p]
    L.shim_oracle_lgndr.argtypes = [i, d, p]
    L.shim_oracle_lgndrgt1.argtypes = [i, d, d, p]
    return L


def tri(n, m):
    return m + n * (n + 1) // 2


def scaled_in(scal, x, nb):
    """sqrt(pi/2x) I_{n+1/2}(x) / scal^n from scipy, with the reference's
    zero above x = 100."""
    if x > 100.0:
        return np.zeros(nb + 1)
    n = np.arange(nb + 1)
    return special.spherical_in(n, x) / scal ** n


@pytest.mark.parametrize("fn", ["shim_engine_bessel_in", "shim_oracle_i_n"])
@pytest.mark.parametrize("nb", [9, 18, 40])
def test_scaled_bessel_in_matches_scipy(shim, fn, nb):
    rng = np.random.default_rng(nb)
    xs = np.concatenate([[2e-4, 1e-3, 0.01, 0.1, 0.5, 1.0, 2.5, 10.0, 37.0, 99.9],
                         10.0 ** rng.uniform(-3.5, 2.0, 40)])
    worst = 0.0
    for x in xs:
        for scal in (1.0, 0.5, 0.1, 0.02):
            b = np.zeros(nb + 1)
            getattr(shim, fn)(scal, float(x), nb, b.ctypes.data)
            ref = scaled_in(scal, x, nb)
            # entries the recurrence zeroes below 1e-300 are compared as zero
            keep = np.abs(ref) > 1e-290
            err = np.abs(b[keep] - ref[keep]) / np.abs(ref[keep])
            worst = max(worst, float(err.max()) if err.size else 0.0)
    assert worst < 1e-12, worst


@pytest.mark.parametrize("fn", ["shim_engine_bessel_in", "shim_oracle_i_n"])
def test_scaled_bessel_in_series_and_cutoff(shim, fn):
    nb = 12
    b = np.zeros(nb + 1)
    for x in (1e-6, 5e-5, 1e-4):
        for scal in (1.0, 0.05):
            getattr(shim, fn)(scal, x, nb, b.ctypes.data)
            ref = scaled_in(scal, x, nb)
            keep = np.abs(ref) > 1e-290
            assert np.allclose(b[keep], ref[keep], rtol=1e-12, atol=0), (x, scal)
    getattr(shim, fn)(0.5, 100.5, nb, b.ctypes.data)
    assert np.all(b == 0.0)


def legendre_gt1_ref(nmax, scal, x):
    """scal^n P_n^m(x) for x > 1 without the Condon-Shortley phase:
    (x^2 - 1)^(m/2) d^m/dx^m P_n(x), from numpy's Legendre series."""
    out = np.zeros((nmax + 1) * (nmax + 2) // 2)
    for n in range(nmax + 1):
        c = np.zeros(n + 1)
        c[n] = 1.0
        for m in range(n + 1):
            dm = npleg.legder(c, m) if m else c
            out[tri(n, m)] = scal ** n * (x * x - 1.0) ** (m / 2) * npleg.legval(x, dm)
    return out


def test_legendre_abs_le_1_matches_scipy(shim):
    nmax = 18
    y = np.zeros((nmax + 1) * (nmax + 2) // 2)
    for x in np.linspace(-0.999, 0.999, 37):
        shim.shim_oracle_lgndr(nmax, float(x), y.ctypes.data)
        for n in range(nmax + 1):
            for m in range(n + 1):
                ref = special.lpmv(m, n, x)  # includes (-1)^m
                scale = factorial(n + m) / factorial(n - m) if m else 1.0
                assert abs(y[tri(n, m)] - ref) <= 1e-11 * max(1.0, abs(ref), scale ** 0.5), (x, n, m)


@pytest.mark.parametrize("fn", ["shim_engine_legendre_gt1", "shim_oracle_lgndrgt1"])
def test_legendre_gt1_matches_series(shim, fn):
    nmax = 9
    y = np.zeros((nmax + 1) * (nmax + 2) // 2)
    for x in (1.0001, 1.05, 1.5, 3.0, 12.0):
        for scal in (1.0, 0.25, 0.05):
            getattr(shim, fn)(nmax, scal, x, y.ctypes.data)
            ref = legendre_gt1_ref(nmax, scal, x)
            assert np.allclose(y, ref, rtol=1e-10, atol=1e-300), (x, scal, np.max(np.abs(y - ref) / np.abs(ref)))
