"""A seeded sweep of small problems against the oracle on the same tree:
sphere or star surfaces of 162-2562 patches, one or two placed instances,
kappa in [0, 0.2], the reference tree at various nbsize or the device tree
at various leaf caps, both engines.  The matvec must match the oracle to
1e-9 (FP64 engine) or 1e-5 (mixed engine, against the FP32-coefficient
oracle), and the right-hand side to 1e-12 / 1e-6."""
import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def case(seed):
    rng = np.random.default_rng(seed)
    k = int(rng.integers(2, 5))
    star = bool(rng.integers(0, 2))
    radius = float(rng.uniform(8.0, 20.0))
    if star:
        V, T, shape = b.star_surface(k, radius, seed=seed)
        mesh = b.Mesh(V, T, b.charges_in_star(int(rng.integers(5, 60)), shape, seed=seed + 1))
    else:
        V, T = b.icosphere(k, radius)
        mesh = b.Mesh(V, T, b.charges_in_sphere(int(rng.integers(5, 60)), 0.7 * radius, seed=seed + 1))
    kappa = float(rng.choice([0.0, rng.uniform(0.02, 0.2)]))
    if rng.integers(0, 2):
        tree = dict(tree="device", leaf_size=int(rng.choice([16, 32, 64, 128])))
    else:
        tree = dict(nbsize=int(rng.choice([50, 100, 300, 1000])))
    two = bool(rng.integers(0, 2))
    return mesh, kappa, tree, two, float(rng.uniform(1.5, 4.0))


@pytest.mark.parametrize("seed", range(900, 912))
def test_random_problem_matches_oracle(seed):
    mesh, kappa, tree, two, eps_in = case(seed)
    ctx = b.EngineContext(0)
    try:
        for precision in ("fp64", "mixed"):
            bp = b.BEEP(kappa=kappa, precision=precision, context=ctx, **tree)
            bp.insert_mesh_instance(mesh, eps_protein=eps_in)
            if two:
                q = b.random_quaternion(np.random.default_rng(seed))
                bp.insert_mesh_instance(mesh, offset=mesh.centre + np.array([3.0, 0.5, -1.0]) * mesh.radius,
                                        rotation=q, eps_protein=eps_in)
            x = np.random.default_rng(seed + 7).standard_normal(2 * bp.num_patches)
            y = bp.matvec(x)
            rhs = bp.set_rhs().copy()
            _, edge = bp.calculate_bounding_cube()
            pr = O.Problem(bp.gathered(), bp.tree(), kappa, fp32=(precision == "mixed"), cube_edge=edge, nterms=9)
            try:
                yo = pr.matvec(x)
                ch = np.concatenate([i.charges for i in bp.instances])
                ro = O.rhs(pr.patches, ch, 80.0)
            finally:
                pr.close()
            bp.close()
            assert rel_l2(y, yo) < (1e-9 if precision == "fp64" else 1e-5), (precision, tree, kappa)
            assert rel_l2(rhs, ro) < (1e-12 if precision == "fp64" else 1e-6), (precision, tree, kappa)
    finally:
        ctx.close()
