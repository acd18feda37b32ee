"""Rigid-body scan and serving loop on the GPU: concurrent solves give the
same results as the same solves run alone."""
import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200.scan import Pose, random_poses, rigid_body_scan
from beep3_b200.server import BemServer, SolveRequest, latency_percentiles

pytestmark = pytest.mark.gpu


def small_star(k, seed, radius=12.0, n_charges=20):
    V, T, shape = b.star_surface(k, radius, seed=seed)
    return b.Mesh(V, T, b.charges_in_star(n_charges, shape, seed=seed + 100))


def test_scan_concurrent_equals_sequential():
    a, c = small_star(3, 1), small_star(3, 2, radius=8.0)
    poses = random_poses(4, seed=3, rmin=25.0, rmax=40.0)
    r1 = rigid_body_scan(a, c, poses, kappa=0.1, workers=1, nbsize=200)
    r3 = rigid_body_scan(a, c, poses, kappa=0.1, workers=3, nbsize=200)
    assert r1.energies == r3.energies  # deterministic kernels: bitwise equal
    assert all(np.isfinite(r1.energies))
    # interaction energy vanishes with separation
    far = rigid_body_scan(a, c, [Pose(np.array([1.0, 0, 0, 0]), np.array([400.0, 0, 0]))], kappa=0.1, workers=1,
                          nbsize=200)
    assert abs(far.energies[0]) < 1e-3 * abs(far.e_a)


def test_server_mix_equals_alone():
    meshes = [small_star(3, s) for s in range(4)] + [small_star(4, 9)]
    kappas = [0.0, 0.05, 0.1, 0.15, 0.1]
    # alone: one at a time
    srv = BemServer(workers=1, nbsize=300)
    alone = [srv.submit(SolveRequest(m, k, tag=i)).result(timeout=300) for i, (m, k) in enumerate(zip(meshes, kappas))]
    srv.close()
    # in the mix: all submitted at once, 3 in flight
    srv = BemServer(workers=3, nbsize=300)
    futs = [srv.submit(SolveRequest(m, k, tag=i)) for i, (m, k) in enumerate(zip(meshes, kappas))]
    mix = [f.result(timeout=300) for f in futs]
    srv.close()
    for a_, m_ in zip(alone, mix):
        assert a_.converged and m_.converged
        assert a_.energy_kj_per_mol == m_.energy_kj_per_mol
    p = latency_percentiles(mix)
    assert p["p99"] >= p["p50"] > 0


def test_far_field_plan_shared_between_problems():
    """A problem whose far-field key (order, kappa, cube edge, levels,
    precision) matches a plan its context keeps adopts it: its results are
    bitwise those of the same problem built on a fresh context, and its
    set-up skips the tables and operators."""
    a = small_star(4, 7, radius=20.0, n_charges=30)
    res = {}
    for precision in ("mixed", "fp64"):
        shared = b.EngineContext(0)
        times = []
        ys = []
        for _ in range(2):
            bp = b.BEEP(kappa=0.1, nbsize=100, precision=precision, context=shared)
            bp.insert_mesh_instance(a)
            inf = bp.info()
            assert inf.fmm_active == 1
            times.append(inf.fmm_setup_ms)
            x = np.random.default_rng(1).standard_normal(2 * bp.num_patches)
            ys.append(bp.matvec(x))
            bp.close()
        fresh = b.BEEP(kappa=0.1, nbsize=100, precision=precision)
        fresh.insert_mesh_instance(a)
        y_fresh = fresh.matvec(x)
        fresh.close()
        shared.close()
        assert np.array_equal(ys[1], ys[0]) and np.array_equal(ys[1], y_fresh)
        res[precision] = times
    assert res["mixed"][1] < res["mixed"][0]


def test_scan_with_snapped_cubes_matches_exact_cubes():
    a, c = small_star(4, 11, radius=20.0, n_charges=30), small_star(3, 12, radius=10.0)
    poses = random_poses(6, seed=5, rmin=35.0, rmax=45.0)
    exact = rigid_body_scan(a, c, poses, kappa=0.1, workers=2, nbsize=150)
    snapped = rigid_body_scan(a, c, poses, kappa=0.1, workers=2, nbsize=150, snap_cube_edges=True)
    ce, cs = np.array(exact.complex_energies), np.array(snapped.complex_energies)
    assert np.max(np.abs(cs - ce) / np.abs(ce)) < 1e-4
