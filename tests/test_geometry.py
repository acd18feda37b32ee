"""Surface discretisation (host): node patches and their point lists."""
import numpy as np
import pytest

import beep3_b200 as b


def test_icosphere_counts_and_orientation():
    for k in range(4):
        V, T = b.icosphere(k, 2.0)
        assert len(V) == 10 * 4 ** k + 2
        assert len(T) == 20 * 4 ** k
        np.testing.assert_allclose(np.linalg.norm(V, axis=1), 2.0)
        n = np.cross(V[T[:, 1]] - V[T[:, 0]], V[T[:, 2]] - V[T[:, 0]])
        assert np.all((n * V[T].mean(axis=1)).sum(axis=1) > 0)


@pytest.mark.parametrize("planar", [True, False])
def test_patch_weights(planar):
    V, T = b.icosphere(2, 5.0)
    ps = b.prepare_patches(V, T, planar=planar, qual_rule=4, quad_rule=0)
    n = ps.n
    assert n == len(V)
    # qualocation weights renormalised to one per patch (node_patch.cpp:221-226)
    np.testing.assert_allclose(np.add.reduceat(ps.qual[:, 6], ps.qual_off[:-1]), 1.0, rtol=1e-12)
    # single quadrature point = centroid with weight = area
    assert ps.quad.shape == (n, 7)
    np.testing.assert_allclose(ps.quad[:, :3], ps.centroid)
    np.testing.assert_allclose(ps.quad[:, 6], ps.area)
    # galerkin weights sum to the patch area
    np.testing.assert_allclose(np.add.reduceat(ps.gal[:, 6], ps.gal_off[:-1]), ps.area, rtol=1e-12)
    # 2 sub-triangles x 4 points per adjacent triangle; valence 5 or 6
    counts = np.diff(ps.qual_off)
    assert set(np.unique(counts)) <= {40, 48}
    np.testing.assert_allclose(np.linalg.norm(ps.normal, axis=1), 1.0)
    if planar:
        # the 4-point rule integrates constants exactly on flat triangles
        np.testing.assert_allclose(ps.area.sum(), ps.planar_area, rtol=1e-12)
    else:
        # curved PN area approaches the sphere's from below the planar one
        assert ps.planar_area < ps.total_area < 4 * np.pi * 25.0
        assert abs(ps.area.sum() - ps.total_area) / ps.total_area < 2e-3


def test_pn_sphere_converges():
    errs = []
    for k in (2, 3, 4):
        V, T = b.icosphere(k, 1.0)
        ps = b.prepare_patches(V, T)
        errs.append(abs(ps.total_area - 4 * np.pi) / (4 * np.pi))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-4


def test_transform_rigid():
    V, T = b.icosphere(1, 3.0)
    ps = b.prepare_patches(V, T)
    q = b.random_quaternion(np.random.default_rng(5))
    R = b.quaternion_matrix(q)
    np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-14)
    moved = ps.transformed(R, np.zeros(3), np.array([1.0, 2.0, 3.0]))
    d0 = np.linalg.norm(ps.centroid[0] - ps.centroid[1])
    d1 = np.linalg.norm(moved.centroid[0] - moved.centroid[1])
    assert abs(d0 - d1) < 1e-12
    np.testing.assert_allclose(np.linalg.norm(moved.qual[:, 3:6], axis=1), 1.0)


def test_star_surface_and_charges():
    V, T, shape = b.star_surface(2, 20.0, seed=7)
    r = np.linalg.norm(V, axis=1)
    assert r.min() > 10 and r.max() < 30
    ch = b.charges_in_star(200, shape, seed=3)
    rr = np.linalg.norm(ch[:, :3], axis=1)
    th = np.arccos(np.clip(ch[:, 2] / rr, -1, 1))
    ph = np.arctan2(ch[:, 1], ch[:, 0])
    assert np.all(rr < 0.8 * shape.r_of(th, ph))
    assert np.all(np.abs(ch[:, 3]) <= 1.0)


def test_bad_mesh_is_rejected():
    V, T = b.icosphere(1, 1.0)
    with pytest.raises(b.BeepError):
        b.prepare_patches(V, T[:-1])  # open surface
    bad = T.copy()
    bad[0, 0] = 10 ** 6
    with pytest.raises(b.BeepError):
        b.prepare_patches(V, bad)
