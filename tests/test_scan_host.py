"""Host side of the scan's warm start (no GPU): the initial guess's layout
over a batch of poses, and, on the oracle, that the isolated molecules'
solutions start a complex's GMRES closer to its solution than zero does."""
import numpy as np

import beep3_b200 as b
import oracle as O
from beep3_b200.scan import _pose_guess, random_poses
from conftest import rel_l2


def test_pose_guess_layout():
    na, nb = 3, 2
    xa = np.arange(2 * na, dtype=float)          # f then h of A
    xb = 100 + np.arange(2 * nb, dtype=float)    # f then h of B
    g = _pose_guess((xa, xb, na, nb), 2)
    f = [0, 1, 2, 100, 101, 0, 1, 2, 100, 101]
    h = [3, 4, 5, 102, 103, 3, 4, 5, 102, 103]
    assert g.tolist() == f + h
    assert _pose_guess((xa, xb, na, nb)).tolist() == [0, 1, 2, 100, 101, 3, 4, 5, 102, 103]


def _oracle_solve(insts, x0=None):
    bp = b.BEEP(kappa=0.1, nbsize=300, precision="mixed")
    for m, off, q in insts:
        bp.insert_mesh_instance(m, offset=off, rotation=q, eps_protein=2.0)
    _, edge = bp.calculate_bounding_cube()
    pr = O.Problem(bp.gathered(), bp.host_tree(), 0.1, True, cube_edge=edge, nterms=9)
    try:
        ch = np.concatenate([i.charges for i in bp.instances])
        rhs = O.rhs(pr.patches, ch, 80.0)
        return pr.solve(rhs, 1e-6, 100, x0=x0)[:2]
    finally:
        pr.close()


def test_isolated_solutions_start_the_complex_closer():
    va, ta, sa = b.star_surface(3, 15.0, seed=611)
    vb, tb, sb = b.star_surface(2, 8.0, seed=612)
    ma = b.Mesh(va, ta, b.charges_in_star(30, sa, seed=613))
    mb = b.Mesh(vb, tb, b.charges_in_star(10, sb, seed=614))
    ident = np.array([1.0, 0.0, 0.0, 0.0])
    xa, _ = _oracle_solve([(ma, ma.centre, ident)])
    xb, _ = _oracle_solve([(mb, mb.centre, ident)])
    pose = random_poses(1, seed=615)[0]
    pose.offset = pose.offset / np.linalg.norm(pose.offset) * 35.0
    insts = [(ma, ma.centre, ident), (mb, ma.centre + pose.offset, pose.rotation)]
    x_cold, its_cold = _oracle_solve(insts)
    x_warm, its_warm = _oracle_solve(insts, _pose_guess((xa, xb, ma.n_patches, mb.n_patches)))
    assert its_warm < its_cold
    assert rel_l2(x_warm, x_cold) < 1e-5
