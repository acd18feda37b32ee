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
