"""GPU parity of the full matvec (near field + plane-wave FMM) and of the
solve against the oracle on trees deep enough for the far field."""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from conftest import make_beep, rel_l2

pytestmark = pytest.mark.gpu

# FP64 engine vs FP64 oracle: same expansions and tables, summation order
# differs; mixed engine (FP32 near field + FP32 FMM) vs the FP64-FMM oracle
# in reference-faithful FP32 near-field mode
TOL_FP64 = 1e-9
TOL_MIXED = 1e-5


def scenario(k=4, radius=10.0, nbsize=100, kappa=0.1, seed=5, star=False):
    if star:
        V, T, shape = b.star_surface(k, radius, seed=seed)
        ch = b.charges_in_star(50, shape, seed=seed + 1)
    else:
        V, T = b.icosphere(k, radius)
        ch = b.charges_in_sphere(20, 0.7 * radius, seed=seed)
    return b.Mesh(V, T, ch), kappa, nbsize


def oracle_for(bp, fp32):
    centre, edge = bp.calculate_bounding_cube()
    return O.Problem(bp.gathered(), bp.tree(), bp.kappa, fp32=fp32, cube_edge=edge, nterms=9)


@pytest.fixture(scope="module", params=[("sphere", 0.1), ("sphere", 0.0), ("star", 0.125)])
def case(request):
    kind, kappa = request.param
    mesh, kappa, nb = scenario(k=4, star=(kind == "star"), kappa=kappa, radius=20.0 if kind == "star" else 10.0)
    return mesh, kappa, nb


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fmm_matvec_parity(case, precision):
    mesh, kappa, nb = case
    bp = make_beep(mesh, kappa=kappa, nbsize=nb, precision=precision)
    inf = bp.info()
    assert inf.fmm_active == 1 and inf.n_levels >= 3
    pr = oracle_for(bp, fp32=(precision == "mixed"))
    rng = np.random.default_rng(11)
    for _ in range(2):
        x = rng.standard_normal(2 * pr.n)
        y = bp.matvec(x)
        yo = pr.matvec(x)
        err = rel_l2(y, yo)
        assert err < (TOL_FP64 if precision == "fp64" else TOL_MIXED), err
        # the far field itself, isolated: engine minus its own near field
    bp.close()
    pr.close()


def test_far_field_alone(case):
    """Far field of the engine (matvec minus the oracle's near field) against
    the oracle's FMM, relative to the far field's own size."""
    mesh, kappa, nb = case
    bp = make_beep(mesh, kappa=kappa, nbsize=nb, precision="fp64")
    pr = oracle_for(bp, fp32=False)
    x = np.random.default_rng(2).standard_normal(2 * pr.n)
    far_gpu = bp.matvec(x) - pr.near(x)
    far_or = pr.far(x)
    assert rel_l2(far_gpu, far_or) < 1e-8
    bp.close()


def test_fmm_solve_and_energy(case):
    mesh, kappa, nb = case
    res = {}
    for precision in ("fp64", "mixed"):
        bp = make_beep(mesh, kappa=kappa, nbsize=nb, precision=precision)
        info = bp.solve(1e-6, 100)
        assert info.converged and info.fmm_active
        e, _ = bp.calculate_energies()
        res[precision] = (bp.x.copy(), e, bp.rhs.copy())
        bp.close()
    # oracle solve on the same tree (FP64)
    bp = make_beep(mesh, kappa=kappa, nbsize=nb)
    pr = oracle_for(bp, fp32=False)
    xo, its, rr = pr.solve(res["fp64"][2], 1e-6, 100)
    assert rel_l2(res["fp64"][0], xo) < 1e-6
    assert rel_l2(res["mixed"][0], xo) < 1e-5
    e64, em = res["fp64"][1], res["mixed"][1]
    assert abs(em - e64) / abs(e64) < 1e-4
    bp.close()


def test_restart_and_device_stream_profile():
    mesh, kappa, nb = scenario(k=4, nbsize=80)
    bp = make_beep(mesh, kappa=kappa, nbsize=nb, precision="mixed")
    import ctypes as C
    import torch
    from beep3_b200 import _native as N
    p = bp.build()
    x = torch.randn(2 * bp.num_patches, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    ms = np.zeros(8)
    launches = np.zeros(8, np.int32)
    ns = C.c_int32()
    N.check(N.lib().bp_matvec_profile(p, x.data_ptr(), y.data_ptr(), 3, N.ptr(ms), N.ptr(launches), C.byref(ns)))
    # near field (the far field is added in its store); P2M one launch; L2P
    # preparation (stage 5) and evaluation (stage 7) one launch each
    assert ns.value == 8 and launches[0] == 1 and launches[1] == 1 and launches[5] == 1 and launches[7] == 1
    assert np.all(ms >= 0) and ms.sum() > 0
    y2 = bp.matvec(x.cpu().numpy())
    assert rel_l2(y.cpu().numpy(), y2) < 1e-12
    bp.close()
