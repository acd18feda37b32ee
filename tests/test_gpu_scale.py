"""Precision at scale: the mixed engine (FP32 near field, FP32 FMM with
3xTF32 tensor-core conversions, FP64 singular terms and GMRES) against the
FP64 engine on a 163842-patch star molecule.  The FP64 engine itself
matches the FP64 oracle to 1e-9 on the smaller trees of test_gpu_fmm.py and
at 40962 patches in test_gpu_configs.py; here the comparison is between
the two engines on the same tree, with the bars of the mixed engine: 1e-5
relative L2 on the matvec and on the solved surface potentials, 1e-4
relative on the solvation energy.  Both engines' matvec rows are also
compared, on 1024 random targets, with the FP64 direct-sum oracle (every
near pair in FP64, the far field summed exactly): the error is the order-9
FMM's truncation, and the mixed engine adds no more than 2e-4 to it."""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from conftest import make_beep, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big_star():
    V, T, shape = b.star_surface(7, 40.0, seed=77)
    return b.Mesh(V, T, b.charges_in_star(20000, shape, seed=78))


@pytest.mark.parametrize("kappa", [0.05, 0.125])
def test_precision_scaling_163842(big_star, kappa):
    res = {}
    x = None
    for precision in ("fp64", "mixed"):
        bp = make_beep(big_star, kappa=kappa, nbsize=1500, precision=precision)
        assert bp.num_patches == 163842
        if x is None:
            x = np.random.default_rng(5).standard_normal(2 * bp.num_patches)
            arr, tree = bp.gathered(), bp.tree()
        y = bp.matvec(x)
        info = bp.solve(1e-6, 100)
        assert info.converged
        e, _ = bp.calculate_energies()
        res[precision] = (y, bp.x.copy(), info.num_iterations, e)
        bp.close()
    y64, x64, it64, e64 = res["fp64"]
    ym, xm, itm, em = res["mixed"]
    assert rel_l2(ym, y64) < 1e-5
    assert rel_l2(xm, x64) < 1e-5
    assert abs(itm - it64) <= 1
    assert abs(em - e64) / abs(e64) < 1e-4
    n = len(x) // 2
    targets = np.random.default_rng(6).choice(n, 1024, replace=False)
    ex = O.exact_rows(arr, tree, kappa, x, targets)
    e64f, e64h = O.row_errors(y64, ex, targets, n)
    emf, emh = O.row_errors(ym, ex, targets, n)
    print(f"kappa {kappa}: matvec rows vs the FP64 direct sum: FP64 engine f {e64f:.3e} h {e64h:.3e}, "
          f"mixed f {emf:.3e} h {emh:.3e}; GMRES iterations {it64}/{itm}; energy mixed vs FP64 "
          f"{abs(em - e64) / abs(e64):.2e}")
    assert e64f < 3e-3 and e64h < 5e-2
    assert abs(emf - e64f) < 2e-4 and abs(emh - e64h) < 2e-4
