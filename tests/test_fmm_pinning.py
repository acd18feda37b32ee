"""The oracle's plane-wave FMM against the direct sum it approximates.

The oracle FMM restates the reference's operators; a shared mistake in that
restatement (a channel sign in FMM_results_to_BEM, an rlsc / xs / ys / zs
table, the i_n recurrence) would pass every engine-vs-oracle test.  So the
oracle's far field is checked here against the exact 12-channel sum over
the same far pairs (src/fmm/test_fmm.cpp:181-214 does the same for the
vanilla FMM), on 4- and 5-level trees, at the matvec's order 9 and at order
18.  Order 9 is the reference's "3 figure" FMM (src/beep/beep.h:123-124): the
potential channels come out near 1e-3, the normal derivative, built from
Hessians, near 2e-2.  At order 18 ("6 figure", src/beep/beep.h:125-126) the
same errors fall by two to three orders of magnitude, which a structural
error would not do: that is the pin.

Bounds are about twice the measured errors.  At kappa = 0 every channel has
the same kernel, the charge terms of channels 3 and 11 cancel exactly in f
and only the dipole terms remain, so f's relative error is that of a field.
"""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O

CASES = {
    # name: (kind, icosphere level, nbsize, kappa)
    "sphere-k0.1": ("sphere", 5, 200, 0.1),
    "sphere-k0": ("sphere", 5, 200, 0.0),
    "star-k0.1": ("star", 5, 150, 0.1),
}
# (f bound, h bound) per order and kappa > 0
BOUNDS = {(9, True): (3e-3, 5e-2), (9, False): (3e-2, 5e-2),
          (18, True): (1.5e-5, 6e-5), (18, False): (6e-5, 6e-5)}


def setup_case(name):
    kind, k, nb, kappa = CASES[name]
    if kind == "star":
        V, T, shape = b.star_surface(k, 20.0, seed=3)
        ch = b.charges_in_star(20, shape, seed=4)
    else:
        V, T = b.icosphere(k, 10.0)
        ch = b.charges_in_sphere(20, 7.0, seed=4)
    bp = b.BEEP(kappa=kappa, nbsize=nb)
    bp.insert_mesh_instance(b.Mesh(V, T, ch))
    arr, tree = bp.gathered(), bp.host_tree()
    _, edge = bp.calculate_bounding_cube()
    return arr, tree, kappa, edge


@pytest.fixture(scope="module", params=list(CASES))
def case(request):
    arr, tree, kappa, edge = setup_case(request.param)
    assert tree["n_levels"] - 1 >= 3  # at least two levels of interaction lists
    n = len(arr["area"])
    x = np.random.default_rng(1).standard_normal(2 * n)
    targets = np.random.default_rng(2).choice(n, 150, replace=False)
    ref = O.direct_far(arr, tree, kappa, x, targets)
    return dict(arr=arr, tree=tree, kappa=kappa, edge=edge, x=x, targets=targets, ref=ref, n=n)


def oracle_far(c, nterms):
    pr = O.Problem(c["arr"], c["tree"], c["kappa"], fp32=False, cube_edge=c["edge"], nterms=nterms)
    try:
        return pr.far(c["x"])
    finally:
        pr.close()


def test_oracle_fmm_converges_to_the_direct_sum(case):
    errs = {}
    for nt in (9, 18):
        errs[nt] = O.row_errors(oracle_far(case, nt), case["ref"], case["targets"], case["n"])
        bf, bh = BOUNDS[(nt, case["kappa"] > 0)]
        assert errs[nt][0] < bf and errs[nt][1] < bh, (nt, errs[nt])
    # more terms: two orders of magnitude or more on both rows
    assert errs[18][0] < errs[9][0] / 100 and errs[18][1] < errs[9][1] / 100, errs
