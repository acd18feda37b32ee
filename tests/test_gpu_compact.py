"""The compact near field (BP_FLAG_COMPACT_NEARFIELD): FP32 coefficients
rounded to 24 bits, 12 bytes a pair.  Each coefficient moves by at most
2^-16 of itself, so the matvec stays within 2e-5 of the FP32-coefficient
path and of the oracle, the solve converges in the same iterations to an
energy within 1e-5, and the problem holds 4 bytes a pair less."""
import ctypes as C

import numpy as np
import pytest

import beep3_b200 as b
import beep3_b200._native as N
import oracle as O
from conftest import make_beep, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["sphere-nofmm", "star-fmm"])
def mesh_case(request):
    if request.param == "sphere-nofmm":
        V, T = b.icosphere(3, 10.0)
        return b.Mesh(V, T, b.charges_in_sphere(10, 7.0, seed=1234)), 1500, 0.1
    V, T, shape = b.star_surface(5, 20.0, seed=5)
    return b.Mesh(V, T, b.charges_in_star(200, shape, seed=6)), 300, 0.1


def test_compact_matches_fp32_coefficients(mesh_case):
    mesh, nb, kappa = mesh_case
    full = make_beep(mesh, kappa=kappa, nbsize=nb, precision="mixed")
    comp = make_beep(mesh, kappa=kappa, nbsize=nb, precision="mixed", compact_nearfield=True)
    i_f, i_c = full.info(), comp.info()
    assert i_f.n_nearfield_pairs == i_c.n_nearfield_pairs
    assert i_f.device_bytes - i_c.device_bytes >= 0.9 * 4 * i_f.n_nearfield_pairs
    x = np.random.default_rng(11).standard_normal(2 * full.num_patches)
    yf, yc = full.matvec(x), comp.matvec(x)
    assert 0 < rel_l2(yc, yf) < 2e-5
    pr = O.Problem(full.gathered(), full.tree(), kappa, fp32=True, cube_edge=full.calculate_bounding_cube()[1],
                   nterms=9)
    try:
        assert rel_l2(yc, pr.matvec(x)) < 2e-5
    finally:
        pr.close()
    s_f, s_c = full.solve(1e-6, 100), comp.solve(1e-6, 100)
    assert s_c.converged and abs(s_f.num_iterations - s_c.num_iterations) <= 1
    e_f, _ = full.calculate_energies()
    e_c, _ = comp.calculate_energies()
    assert abs(e_c - e_f) / abs(e_f) < 1e-5
    full.close()
    comp.close()


def test_compact_gather_path():
    """A neighbourhood wider than the apply kernel's x staging (one leaf of
    40962 patches) reads the compact planes through the gather path."""
    V, T = b.icosphere(6, 20.0)
    mesh = b.Mesh(V, T, b.charges_in_sphere(40, 15.0, seed=77))
    ctx = b.EngineContext(0)
    try:
        x = np.random.default_rng(5).standard_normal(2 * mesh.n_patches)
        ys = []
        for compact in (False, True):
            bp = b.BEEP(kappa=0.1, nbsize=40962, precision="mixed", context=ctx, compact_nearfield=compact)
            bp.insert_mesh_instance(mesh)
            inf = bp.info()
            assert inf.n_leaves == 1 and inf.n_nearfield_cols == 40962
            ys.append(bp.matvec(x))
            bp.close()
        assert 0 < rel_l2(ys[1], ys[0]) < 2e-5
    finally:
        ctx.close()


def test_compact_flag_rejected_off_the_mixed_cached_path():
    V, T = b.icosphere(2, 10.0)
    mesh = b.Mesh(V, T, b.charges_in_sphere(5, 7.0, seed=3))
    with pytest.raises(ValueError):
        b.BEEP(precision="fp64", compact_nearfield=True)
    with pytest.raises(ValueError):
        b.BEEP(precision="mixed", nearfield_on_demand=True, compact_nearfield=True)
    bp = make_beep(mesh, kappa=0.1, nbsize=100, precision="mixed", compact_nearfield=True)
    bp.build()
    centre, edge = bp.calculate_bounding_cube()
    insts = (N.bp_instance * 1)()
    insts[0].mesh = bp._mesh_handle(mesh)
    insts[0].rotation[:] = [1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0]
    insts[0].offset[:] = [0.0, 0.0, 0.0]
    insts[0].dielectric_ratio = 2.0 / 80.0
    h = C.c_void_p()
    for prec, extra in ((N.BP_PREC_FP64, 0), (N.BP_PREC_MIXED, N.BP_FLAG_NEARFIELD_ON_DEMAND)):
        prm = N.bp_params(0.1, 1e-10, (C.c_double * 3)(*centre), edge, 100, 9, prec,
                          N.BP_FLAG_COMPACT_NEARFIELD | extra)
        assert N.lib().bp_problem_create_posed(bp.context(), insts, 1, C.byref(prm), C.byref(h)) == N.BP_ERR_INVALID
        assert b"compact near field" in N.lib().bp_last_error()
    bp.close()
