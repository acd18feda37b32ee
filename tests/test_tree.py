"""The engine's adaptive octree (host, C++) against the pure-Python
restatement of the reference rules, plus structural invariants."""
import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200.beep import build_tree
from conftest import make_beep
from oracle import tree as OT


def scenario(k, nbsize, star=False, seed=3):
    if star:
        V, T, shape = b.star_surface(k, 20.0, seed=seed)
        ch = b.charges_in_star(20, shape, seed=seed)
    else:
        V, T = b.icosphere(k, 10.0)
        ch = b.charges_in_sphere(10, 7.0, seed=seed)
    bp = make_beep(b.Mesh(V, T, ch), nbsize=nbsize)
    pts = bp.gathered()["centroid"]
    centre, edge = bp.calculate_bounding_cube()
    return pts, centre, edge


@pytest.mark.parametrize("k,nbsize,star", [(3, 60, False), (3, 200, False), (4, 100, False), (4, 300, True),
                                           (3, 1500, False)])
def test_tree_matches_python_restatement(k, nbsize, star):
    pts, centre, edge = scenario(k, nbsize, star)
    t = build_tree(pts, centre, edge, nbsize)
    r = OT.build(pts, centre, edge, nbsize)
    assert t["n_levels"] == r["n_levels"]
    np.testing.assert_array_equal(t["info"], r["info"])
    np.testing.assert_allclose(t["geom"], r["geom"], rtol=0, atol=1e-12)
    np.testing.assert_array_equal(t["contents"], r["contents"])


@pytest.mark.parametrize("k,nbsize", [(4, 100), (5, 400)])
def test_tree_invariants(k, nbsize):
    pts, centre, edge = scenario(k, nbsize)
    t = build_tree(pts, centre, edge, nbsize)
    info, contents = t["info"], t["contents"]
    n = len(pts)
    leaf = (info[:, 4] & 2) > 0
    shadow = (info[:, 4] & 4) > 0
    assert not np.any(leaf & shadow)
    # leaves partition the patches
    seen = np.zeros(n, int)
    for r in info[leaf]:
        seen[contents[r[6]:r[6] + r[7]]] += 1
    assert np.all(seen == 1)
    # every patch lies in its node's cube
    for k_, r in enumerate(info):
        c, e = t["geom"][k_, :3], t["geom"][k_, 3]
        p = pts[contents[r[6]:r[6] + r[7]]]
        if len(p):
            assert np.all(np.abs(p - c) <= e / 2 * (1 + 1e-9))
    # mean explicit work per item within the target (BEEP's nbsize rule)
    key = {(int(r[0]), int(r[1]), int(r[2]), int(r[3])): int(r[7]) for r in info}
    work = 0
    for r in info[leaf]:
        L, x, y, z = (int(v) for v in r[:4])
        nb = sum(key.get((L, x + dx, y + dy, z + dz), 0) for dx in (-1, 0, 1) for dy in (-1, 0, 1)
                 for dz in (-1, 0, 1))
        work += nb * int(r[7])
    assert work / n <= nbsize * 1.05
    # children of split non-shadow nodes' neighbours exist (full neighbourhoods)
    assert t["n_levels"] >= 3


@pytest.mark.parametrize("nbsize", [60, 100, 200])
def test_tree_ties_on_split_planes(nbsize):
    """Points on a lattice whose planes are the nodes' split planes (the
    child choice p > centre sends ties to the lower child), with duplicates:
    the C++ tree has the restatement's nodes, parents, children and
    contents.  Leaf flags and local-expansion slots are left out: on a
    lattice many leaves tie on their neighbourhood count, and which of them
    the refinement splits follows the sort's order of ties (std::sort in the
    engine, as in the reference; a stable sort in the restatement)."""
    g = np.arange(-8.0, 8.01, 2.0)
    pts = np.array([[x, y, z] for x in g for y in g for z in g])
    pts = np.concatenate([pts, pts[::7]])  # duplicated points
    t = build_tree(pts, np.zeros(3), 16.0, nbsize)
    r = OT.build(pts, np.zeros(3), 16.0, nbsize)
    assert t["n_levels"] == r["n_levels"]
    cols = [0, 1, 2, 3, 5, 6, 7, 8] + list(range(10, 18))
    np.testing.assert_array_equal(t["info"][:, cols], r["info"][:, cols])
    np.testing.assert_array_equal(t["contents"], r["contents"])


@pytest.mark.parametrize("k,cap,star", [(4, 16, False), (4, 64, True), (5, 64, True), (3, 1, False)])
def test_leaf_capped_restatement_invariants(k, cap, star):
    """The device-tree mode's rule, restated: leaves hold at most `cap`
    points (or sit at depth 20), every existing neighbour of a node split by
    size has children, shadows are never leaves, and the leaves partition
    the points, each inside its leaf's cell."""
    pts, centre, edge = scenario(k, 100, star)
    t = OT.build_leaf_capped(pts, centre, edge, cap)
    info, geom, contents = t["info"], t["geom"], t["contents"]
    n = len(pts)
    has_ch, leaf, shadow = (info[:, 4] & 1) > 0, (info[:, 4] & 2) > 0, (info[:, 4] & 4) > 0
    assert not np.any(leaf & shadow)
    assert np.all((info[leaf, 7] <= cap) | (info[leaf, 0] == OT.DEPTH) | has_ch[leaf])
    seen = np.zeros(n, int)
    for r, g in zip(info[leaf], geom[leaf]):
        items = contents[r[6]:r[6] + r[7]]
        seen[items] += 1
        assert np.all(np.abs(pts[items] - g[:3]) <= g[3] / 2 * (1 + 1e-12))
    assert np.all(seen == 1)
    at = {(r[0], r[1], r[2], r[3]): j for j, r in enumerate(info)}
    for j, r in enumerate(info):
        split_by_size = has_ch[j] and not leaf[j] and not shadow[j]
        if not split_by_size:
            continue
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    m = at.get((r[0], r[1] + dx, r[2] + dy, r[3] + dz))
                    if m is not None:
                        assert has_ch[m]
    # children of a split leaf (a neighbour split) are shadows; of a node
    # split by size, not
    for j, r in enumerate(info):
        for c in r[10:18]:
            if c >= 0:
                assert info[c, 5] == j
                assert shadow[c] == (shadow[j] or leaf[j])
