"""The GPU engine checked against results it shares no code with.

* The analytic Kirkwood series for charges in a dielectric sphere with salt,
  on a 10242-patch sphere whose tree is deep enough for the plane-wave FMM
  (the 642-patch Kirkwood case of test_gpu_nearfield.py has no far field).
  The BEM discretisation error of the PN sphere is about 1e-3 at this size
  and about 2e-3 at 2562 patches (measured with the oracle; the FMM order
  moves the energy by about 5e-5), so the bound is 2e-3 and the error must
  shrink from 2562 to 10242 patches.
* The far field (matvec minus the oracle's near field) against the exact
  12-channel sum over the same far pairs on 150 targets, the method of the
  reference's own FMM self-check (src/fmm/test_fmm.cpp:181-214).  The
  order-9 FMM is a "3 figure" method (src/beep/beep.h:123-124); the bounds
  are those of the oracle's own FMM (tests/test_fmm_pinning.py, which also
  shows the oracle converging to the direct sum at order 18), and the engine
  must not add measurable error to the truncation: its errors equal the
  oracle FMM's within 1e-4 (FP64 engine) and 2e-4 (mixed engine).
"""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from conftest import make_beep, rel_l2
from oracle import kirkwood as K

pytestmark = pytest.mark.gpu


def kirkwood_energy(k, nbsize, kappa, precision):
    V, T = b.icosphere(k, 10.0)
    mesh = b.Mesh(V, T, b.charges_in_sphere(10, 7.0, seed=1234))
    bp = make_beep(mesh, kappa=kappa, nbsize=nbsize, precision=precision)
    inf = bp.info()
    assert inf.fmm_active == 1 and inf.n_levels >= 4
    info = bp.solve(1e-6, 100)
    assert info.converged
    e, _ = bp.calculate_energies()
    inst = bp.instances[0]
    ek = K.solvation_energy(inst.charges, 10.0, 2.0, 80.0, kappa, centre=inst.offset)
    bp.close()
    return e, ek


@pytest.mark.parametrize("kappa", [0.1, 0.0])
def test_kirkwood_with_fmm_active(kappa):
    res = {p: kirkwood_energy(5, 300, kappa, p) for p in ("fp64", "mixed")}
    ek = res["fp64"][1]
    err = {p: abs(res[p][0] - ek) / abs(ek) for p in res}
    assert err["fp64"] < 2e-3 and err["mixed"] < 2e-3, err
    assert abs(res["mixed"][0] - res["fp64"][0]) / abs(res["fp64"][0]) < 1e-4
    # discretisation convergence: the coarser sphere is further off
    e4, _ = kirkwood_energy(4, 100, kappa, "fp64")
    assert abs(e4 - ek) / abs(ek) > err["fp64"]


CASES = {
    "sphere-k0.1": ("sphere", 5, 200, 0.1),
    "sphere-k0": ("sphere", 5, 200, 0.0),
    "star-k0.1": ("star", 5, 150, 0.1),
}
BOUNDS = {True: (3e-3, 5e-2), False: (3e-2, 5e-2)}  # order 9, kappa > 0 / kappa = 0


@pytest.fixture(scope="module", params=list(CASES))
def far_case(request):
    kind, k, nb, kappa = CASES[request.param]
    if kind == "star":
        V, T, shape = b.star_surface(k, 20.0, seed=3)
        ch = b.charges_in_star(20, shape, seed=4)
    else:
        V, T = b.icosphere(k, 10.0)
        ch = b.charges_in_sphere(20, 7.0, seed=4)
    return b.Mesh(V, T, ch), nb, kappa


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_engine_far_field_matches_direct_sum(far_case, precision):
    mesh, nb, kappa = far_case
    bp = make_beep(mesh, kappa=kappa, nbsize=nb, precision=precision)
    assert bp.info().fmm_active == 1
    arr, tree = bp.gathered(), bp.tree()
    _, edge = bp.calculate_bounding_cube()
    n = bp.num_patches
    x = np.random.default_rng(1).standard_normal(2 * n)
    targets = np.random.default_rng(2).choice(n, 150, replace=False)
    pr = O.Problem(arr, tree, kappa, fp32=(precision == "mixed"), cube_edge=edge, nterms=9)
    far_gpu = bp.matvec(x) - pr.near(x)
    far_or = pr.far(x)
    pr.close()
    bp.close()
    ref = O.direct_far(arr, tree, kappa, x, targets)
    e_gpu = O.row_errors(far_gpu, ref, targets, n)
    e_or = O.row_errors(far_or, ref, targets, n)
    bf, bh = BOUNDS[kappa > 0]
    assert e_gpu[0] < bf and e_gpu[1] < bh, e_gpu
    slack = 1e-4 if precision == "fp64" else 2e-4
    assert abs(e_gpu[0] - e_or[0]) < slack and abs(e_gpu[1] - e_or[1]) < slack, (e_gpu, e_or)
