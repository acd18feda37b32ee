"""Parity at the benchmark's own configuration: the 40962-patch star
molecule (2000 charges, kappa 0.1, the reference's tree at nbsize 1500, FMM
order 9), both engines against the oracle on the same tree.

Bars: the FP64 engine matches the FP64 oracle to 1e-9 on the matvec; the
mixed engine matches the reference-faithful oracle (FP32 near-field
coefficients, FP64 FMM) to 1e-5 on the matvec and on the solved surface
potentials f/h, and both engines' solvation energies match the oracle's to
1e-4 (each engine against the oracle solve from the oracle's own
right-hand side and energy coefficients).  The same matvec rows are also
compared, on 1024 random targets, with the FP64 direct-sum oracle (every
near pair in FP64 and the far field summed exactly), which measures the
order-9 FMM's truncation: both engines must show the oracle FMM's error.
"""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from conftest import make_beep, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def star_s():
    V, T, shape = b.star_surface(6, 20.0, seed=1235)
    return b.Mesh(V, T, b.charges_in_star(2000, shape, seed=1236))


def oracle_solve(pr, arr, inst, mesh):
    rhs = O.rhs(pr.patches, inst.charges, 80.0)
    x, its, _ = pr.solve(rhs, 1e-6, 100)
    ecf, ech = O.energy_coefficients(arr["gal_off"], arr["gal"], arr["area"], inst.charges, mesh.patches.total_area)
    return x, its, O.energy(x[:pr.n], x[pr.n:], ecf, ech, inst.dielectric_ratio)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config_s_matches_the_oracle(star_s, precision):
    bp = make_beep(star_s, kappa=0.1, nbsize=1500, precision=precision)
    assert bp.num_patches == 40962 and bp.info().fmm_active == 1
    arr, tree = bp.gathered(), bp.tree()
    _, edge = bp.calculate_bounding_cube()
    n = bp.num_patches
    x = np.random.default_rng(5).standard_normal(2 * n)
    y = bp.matvec(x)
    info = bp.solve(1e-6, 100)
    assert info.converged
    e, _ = bp.calculate_energies()
    xs = bp.x.copy()
    inst = bp.instances[0]
    bp.close()
    pr = O.Problem(arr, tree, 0.1, fp32=(precision == "mixed"), cube_edge=edge, nterms=9)
    try:
        yo = pr.matvec(x)
        xo, its_o, eo = oracle_solve(pr, arr, inst, star_s)
    finally:
        pr.close()
    assert rel_l2(y, yo) < (1e-9 if precision == "fp64" else 1e-5)
    assert rel_l2(xs, xo) < (1e-7 if precision == "fp64" else 1e-5)
    assert rel_l2(xs[:n], xo[:n]) < 1e-5 and rel_l2(xs[n:], xo[n:]) < 1e-5
    assert abs(e - eo) / abs(eo) < 1e-4
    assert abs(info.num_iterations - its_o) <= 1
    # the same rows against the FP64 direct sum: the order-9 truncation
    targets = np.random.default_rng(6).choice(n, 1024, replace=False)
    ex = O.exact_rows(arr, tree, 0.1, x, targets)
    ef, eh = O.row_errors(y, ex, targets, n)
    of, oh = O.row_errors(yo, ex, targets, n)
    assert ef < 3e-3 and eh < 5e-2, (ef, eh)
    assert abs(ef - of) < 2e-4 and abs(eh - oh) < 2e-4, ((ef, eh), (of, oh))
