"""The near field computed in every matvec (no cached coefficients, the
reference's uncached GPU path) against the cached near field and the oracle:
the same pairs and point lists, so the FP64 engine agrees to rounding
(1e-12) and the mixed engine to its FP32 rounding (1e-6 between the two
paths, 1e-5 against the reference-faithful oracle); the problem holds no
coefficient block."""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from conftest import make_beep, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["sphere-nofmm", "star-fmm"])
def mesh_case(request):
    if request.param == "sphere-nofmm":
        V, T = b.icosphere(3, 10.0)
        return b.Mesh(V, T, b.charges_in_sphere(10, 7.0, seed=1234)), 1500, 0.1
    V, T, shape = b.star_surface(4, 20.0, seed=5)
    return b.Mesh(V, T, b.charges_in_star(50, shape, seed=6)), 100, 0.125


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_on_demand_equals_cached(mesh_case, precision):
    mesh, nb, kappa = mesh_case
    cached = make_beep(mesh, kappa=kappa, nbsize=nb, precision=precision)
    ondem = make_beep(mesh, kappa=kappa, nbsize=nb, precision=precision, nearfield_on_demand=True)
    ic, io = cached.info(), ondem.info()
    assert ic.n_nearfield_pairs == io.n_nearfield_pairs
    coef_bytes = ic.n_nearfield_pairs * (16 if precision == "mixed" else 32)
    assert ic.device_bytes - io.device_bytes >= 0.9 * coef_bytes
    x = np.random.default_rng(3).standard_normal(2 * cached.num_patches)
    yc, yo = cached.matvec(x), ondem.matvec(x)
    assert rel_l2(yo, yc) < (1e-12 if precision == "fp64" else 1e-6)
    pr = O.Problem(cached.gathered(), cached.tree(), kappa, fp32=(precision == "mixed"),
                   cube_edge=cached.calculate_bounding_cube()[1], nterms=9)
    assert rel_l2(yo, pr.matvec(x)) < (1e-9 if precision == "fp64" else 1e-5)
    pr.close()
    # a full solve on the on-demand path
    i1, i2 = cached.solve(1e-6, 100), ondem.solve(1e-6, 100)
    assert i2.converged and abs(i1.num_iterations - i2.num_iterations) <= 1
    e1, _ = cached.calculate_energies()
    e2, _ = ondem.calculate_energies()
    assert abs(e2 - e1) / abs(e1) < 1e-6
    cached.close()
    ondem.close()


def test_oversized_neighbourhood_gathers_x():
    """One leaf of 40962 patches: its 40962 columns exceed the apply
    kernel's shared-memory staging (29056 in FP32), so the cached apply
    gathers x through the column ids; it must equal the on-demand path."""
    V, T = b.icosphere(6, 20.0)
    mesh = b.Mesh(V, T, b.charges_in_sphere(40, 15.0, seed=77))
    cached = make_beep(mesh, kappa=0.1, nbsize=40962, precision="mixed")
    inf = cached.info()
    assert inf.n_leaves == 1 and inf.n_nearfield_cols == 40962 and inf.fmm_active == 0
    x = np.random.default_rng(11).standard_normal(2 * cached.num_patches)
    yc = cached.matvec(x)
    cached.close()
    ondem = make_beep(mesh, kappa=0.1, nbsize=40962, precision="mixed", nearfield_on_demand=True)
    yo = ondem.matvec(x)
    ondem.close()
    assert rel_l2(yc, yo) < 1e-6
