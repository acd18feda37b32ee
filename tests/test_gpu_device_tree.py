"""The octree built on the device (Morton codes, radix sort, per-level
segmentation; BP_FLAG_DEVICE_TREE) against the Python restatement of its
leaf-cap rule, node for node; the matvec on that tree against the oracle on
the same tree; and the device-tree problem against the reference-tree
problem (different near/far splits, so they agree to the order-9 FMM's
accuracy, not to rounding)."""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from conftest import make_beep, rel_l2
from oracle import tree as OT

pytestmark = pytest.mark.gpu


def star(k, n_charges, seed):
    V, T, shape = b.star_surface(k, 20.0, seed=seed)
    return b.Mesh(V, T, b.charges_in_star(n_charges, shape, seed=seed + 1))


@pytest.mark.parametrize("k,cap", [(3, 8), (4, 16), (5, 64), (5, 200)])
def test_device_tree_matches_restatement(k, cap):
    bp = make_beep(star(k, 20, 40 + k), tree="device", leaf_size=cap)
    t = bp.tree()
    centre, edge = bp.calculate_bounding_cube()
    r = OT.build_leaf_capped(bp.gathered()["centroid"], centre, edge, cap)
    bp.close()
    assert t["n_levels"] == r["n_levels"]
    np.testing.assert_array_equal(t["info"], r["info"])
    np.testing.assert_allclose(t["geom"], r["geom"], rtol=0, atol=1e-12 * edge)
    np.testing.assert_array_equal(t["contents"], r["contents"])


def test_device_tree_two_instances():
    """Two meshes apart in one cube: clusters with empty space between."""
    V, T, shape = b.star_surface(4, 20.0, seed=11)
    m = b.Mesh(V, T, b.charges_in_star(30, shape, seed=12))
    bp = b.BEEP(kappa=0.1, tree="device", leaf_size=32)
    bp.insert_mesh_instance(m, offset=(-30.0, 0.0, 0.0))
    bp.insert_mesh_instance(m, offset=(30.0, 5.0, -2.0))
    t = bp.tree()
    centre, edge = bp.calculate_bounding_cube()
    r = OT.build_leaf_capped(bp.gathered()["centroid"], centre, edge, 32)
    bp.close()
    np.testing.assert_array_equal(t["info"], r["info"])
    np.testing.assert_array_equal(t["contents"], r["contents"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_tree_matvec_matches_oracle(precision):
    mesh = star(5, 200, 61)
    bp = make_beep(mesh, kappa=0.125, tree="device", leaf_size=64, precision=precision)
    assert bp.info().fmm_active == 1
    x = np.random.default_rng(8).standard_normal(2 * bp.num_patches)
    y = bp.matvec(x)
    pr = O.Problem(bp.gathered(), bp.tree(), 0.125, fp32=(precision == "mixed"),
                   cube_edge=bp.calculate_bounding_cube()[1], nterms=9)
    bp.close()
    try:
        yo = pr.matvec(x)
    finally:
        pr.close()
    assert rel_l2(y, yo) < (1e-9 if precision == "fp64" else 1e-5)


def test_device_tree_agrees_with_reference_tree():
    """Same scenario, two trees: matvec within the order-9 FMM's error, and
    the solved energy to 1e-4."""
    mesh = star(5, 200, 71)
    ref = make_beep(mesh, kappa=0.1, nbsize=300)
    dev = make_beep(mesh, kappa=0.1, tree="device", leaf_size=64)
    assert ref.info().n_nearfield_pairs != dev.info().n_nearfield_pairs
    x = np.random.default_rng(9).standard_normal(2 * ref.num_patches)
    assert rel_l2(dev.matvec(x), ref.matvec(x)) < 1e-4
    assert ref.solve(1e-6, 100).converged and dev.solve(1e-6, 100).converged
    e_ref, e_dev = ref.calculate_energies()[0], dev.calculate_energies()[0]
    ref.close()
    dev.close()
    assert abs(e_dev - e_ref) < 1e-4 * abs(e_ref)
