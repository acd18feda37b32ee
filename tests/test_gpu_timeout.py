"""The bounded-wait timeout path of the tensor-core FMM kernels, made to run
without breaking anything: with bp_problem_test_wait_timeout switched on,
every CTA of the mixed engine's tensor-core GEMMs also waits on a barrier
that nothing arrives on, with a short bound, so the wait runs out.  The
kernel then stops issuing, drains the MMAs it issued, frees its tensor
memory and flags the problem; the matvec or solve returns BP_ERR_TIMEOUT
once, and the same problem computes correct results again once the switch
is off.  No GPU fault is involved: every wait ends by its bound."""
import ctypes as C

import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200 import _native as N
from conftest import make_beep

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed_fmm_problem():
    V, T = b.icosphere(4, 10.0)
    bp = make_beep(b.Mesh(V, T, b.charges_in_sphere(20, 7.0, seed=5)), kappa=0.1, nbsize=100, precision="mixed")
    assert bp.info().fmm_active == 1
    yield bp
    bp.close()


def test_matvec_reports_timeout_then_recovers(mixed_fmm_problem):
    bp = mixed_fmm_problem
    L = N.lib()
    p = bp.build()
    n2 = 2 * bp.num_patches
    x = np.random.default_rng(3).standard_normal(n2)
    y_ref = bp.matvec(x)
    y = np.empty(n2)
    N.check(L.bp_problem_test_wait_timeout(p, 1))
    try:
        for _ in range(2):  # reported on every matvec that timed out
            assert L.bp_matvec(p, N.ptr(x), N.ptr(y)) == N.BP_ERR_TIMEOUT
            assert b"timed out" in L.bp_last_error()
    finally:
        N.check(L.bp_problem_test_wait_timeout(p, 0))
    # the context and the problem are still usable and the result is the same
    y2 = bp.matvec(x)
    assert np.array_equal(y2, y_ref)


def test_solve_reports_timeout_then_recovers(mixed_fmm_problem):
    bp = mixed_fmm_problem
    L = N.lib()
    p = bp.build()
    bp.set_rhs()
    n2 = 2 * bp.num_patches
    x = np.zeros(n2)
    its, rr = C.c_int32(), C.c_double()
    N.check(L.bp_problem_test_wait_timeout(p, 1))
    try:
        code = L.bp_solve(p, N.ptr(bp.rhs), N.ptr(x), 1e-6, 100, 0, C.byref(its), C.byref(rr))
        assert code == N.BP_ERR_TIMEOUT
    finally:
        N.check(L.bp_problem_test_wait_timeout(p, 0))
    info = bp.solve(1e-6, 100)
    assert info.converged


def test_switch_needs_tensor_core_kernels():
    V, T = b.icosphere(4, 10.0)
    bp = make_beep(b.Mesh(V, T, b.charges_in_sphere(20, 7.0, seed=5)), kappa=0.1, nbsize=100, precision="fp64")
    assert N.lib().bp_problem_test_wait_timeout(bp.build(), 1) == N.BP_ERR_UNSUPPORTED
    bp.close()
