"""Batch problems (bp_problem_create_batch / ScenarioBatch): independent
scenarios in one problem, one forest of trees with a shared cube edge, a
block-diagonal matvec and one GMRES per scenario in shared launches.

Each scenario is compared with its own problem built on the same cube
(BEEP.set_bounding_cube with the batch's edge): the matvec blocks agree to
rounding, GMRES takes the same iterations, and the solvation energies agree
to 1e-6; a scenario that converges early sits out the other scenarios'
steps."""
import numpy as np
import pytest

import beep3_b200 as b
import beep3_b200.scan  # noqa: F401  (b.scan)
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def meshes():
    va, ta, sa = b.star_surface(4, 20.0, seed=301)
    vb, tb, sb = b.star_surface(3, 12.0, seed=302)
    ma = b.Mesh(va, ta, b.charges_in_star(60, sa, seed=303))
    mb = b.Mesh(vb, tb, b.charges_in_star(20, sb, seed=304))
    return ma, mb


def scenarios(meshes, precision, ctx, n=3, lone_sphere=False, **kw):
    ma, mb = meshes
    poses = b.scan.random_poses(n, seed=305, rmin=30.0, rmax=45.0)
    out = []
    for p in poses:
        bp = b.BEEP(kappa=0.1, nbsize=100, precision=precision, context=ctx, **kw)
        bp.insert_mesh_instance(ma, offset=ma.centre, eps_protein=2.0)
        bp.insert_mesh_instance(mb, offset=ma.centre + p.offset, rotation=p.rotation, eps_protein=2.0)
        out.append(bp)
    if lone_sphere:
        V, T = b.icosphere(3, 10.0)
        bp = b.BEEP(kappa=0.1, nbsize=100, precision=precision, context=ctx, **kw)
        bp.insert_mesh_instance(b.Mesh(V, T, b.charges_in_sphere(10, 7.0, seed=306)), eps_protein=2.0)
        out.append(bp)
    return out


def own_problem(scen, centre, edge, precision, ctx, kappa=0.1, **kw):
    bp = b.BEEP(kappa=kappa, nbsize=100, precision=precision, context=ctx, **kw)
    for inst in scen.instances:
        bp.insert_mesh_instance(inst.mesh, offset=inst.offset, rotation=inst.rotation, eps_protein=inst.eps_protein)
    bp.set_bounding_cube(centre, edge)
    return bp


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_blocks_equal_own_problems(meshes, precision):
    ctx = b.EngineContext(0)
    scen = scenarios(meshes, precision, ctx, lone_sphere=True)
    batch = b.ScenarioBatch(scen, context=ctx)
    inf = batch.info()
    assert inf.n_scenarios == len(scen) and inf.fmm_active == 1
    x = np.random.default_rng(7).standard_normal(2 * batch.num_patches)
    y = batch.matvec(x)
    sol = batch.solve(1e-6, 100)
    assert all(sol.converged)
    energies = batch.calculate_energies()
    assert batch.info().gmres_graph == 1
    for k, s in enumerate(scen):
        own = own_problem(s, batch.centres[k], batch.cube_edge, precision, ctx)
        yk = own.matvec(batch.scenario_part(x, k))
        assert rel_l2(batch.scenario_part(y, k), yk) < (1e-12 if precision == "fp64" else 1e-6)
        info = own.solve(1e-6, 100)
        e, per = own.calculate_energies()
        assert info.num_iterations == sol.iterations[k]
        assert abs(energies[k][0] - e) < 1e-6 * abs(e)
        np.testing.assert_allclose(energies[k][1], per, rtol=1e-6)
        own.close()
    # the lone sphere converges in fewer steps than the complexes
    assert sol.iterations[-1] < max(sol.iterations[:-1])
    batch.close()
    ctx.close()


def test_batch_of_device_trees(meshes):
    ctx = b.EngineContext(0)
    scen = scenarios(meshes, "mixed", ctx, n=4, tree="device", leaf_size=48)
    batch = b.ScenarioBatch(scen, context=ctx)
    x = np.random.default_rng(8).standard_normal(2 * batch.num_patches)
    y = batch.matvec(x)
    for k, s in enumerate(scen):
        own = own_problem(s, batch.centres[k], batch.cube_edge, "mixed", ctx, tree="device", leaf_size=48)
        assert rel_l2(batch.scenario_part(y, k), own.matvec(batch.scenario_part(x, k))) < 1e-6
        own.close()
    batch.close()
    ctx.close()


def test_batched_scan_matches_unbatched(meshes):
    """The scan in batches of 4 against pose by pose: complex energies to the
    FMM's truncation error (the batch's cube is larger than a pose's own)."""
    ma, mb = meshes
    poses = b.scan.random_poses(8, seed=310, rmin=30.0, rmax=50.0)
    one = b.scan.rigid_body_scan(ma, mb, poses, kappa=0.1, nbsize=100, workers=2)
    bat = b.scan.rigid_body_scan(ma, mb, poses, kappa=0.1, nbsize=100, workers=2, batch=4)
    np.testing.assert_allclose(bat.complex_energies, one.complex_energies, rtol=2e-4)
    assert abs(bat.e_a - one.e_a) < 1e-9 * abs(one.e_a)


def test_many_scenarios_with_restarts():
    """24 one-sphere scenarios of different sizes, charges and permittivities, solved with
    restarted GMRES (cycles of 4 steps): more scenarios than the dot-product
    blocks of a single problem's solve are split into, and scenarios that
    converge in an early cycle sit out the later ones.  Each matches its own
    problem's restarted solve."""
    ctx = b.EngineContext(0)
    scen = []
    for k in range(24):
        V, T = b.icosphere(2 + k % 2, 8.0 + k)
        bp = b.BEEP(kappa=0.1, nbsize=100, precision="fp64", context=ctx)
        bp.insert_mesh_instance(b.Mesh(V, T, b.charges_in_sphere(3 + k, 5.0 + 0.5 * k, seed=500 + k)),
                                offset=(40.0 * k, 0.0, 0.0), eps_protein=2.0 + 0.1 * k)
        scen.append(bp)
    batch = b.ScenarioBatch(scen, context=ctx)
    assert batch.info().n_scenarios == 24
    sol = batch.solve(1e-8, 200, restart=4)
    assert all(sol.converged)
    energies = batch.calculate_energies()
    its = []
    for k, s in enumerate(scen):
        own = own_problem(s, batch.centres[k], batch.cube_edge, "fp64", ctx)
        info = own.solve(1e-8, 200, restart=4)
        e, _ = own.calculate_energies()
        its.append(info.num_iterations)
        assert info.num_iterations == sol.iterations[k]
        assert abs(energies[k][0] - e) < 1e-9 * abs(e)
        own.close()
    assert len(set(its)) > 1  # the scenarios stop at different steps
    batch.close()
    ctx.close()


def test_batch_iteration_limit_reports_per_scenario():
    """A step limit below what the complexes need: bp_solve_batch returns
    BP_ERR_NOT_CONVERGED and per-scenario residuals above the tolerance."""
    import ctypes as C
    from beep3_b200 import _native as N
    V, T, shape = b.star_surface(3, 15.0, seed=520)
    m = b.Mesh(V, T, b.charges_in_star(20, shape, seed=521))
    ctx = b.EngineContext(0)
    scen = []
    for k in range(3):
        bp = b.BEEP(kappa=0.1, nbsize=100, context=ctx)
        bp.insert_mesh_instance(m, offset=(60.0 * k, 0.0, 0.0), eps_protein=2.0)
        scen.append(bp)
    batch = b.ScenarioBatch(scen, context=ctx)
    rhs = batch.set_rhs()
    x = np.zeros_like(rhs)
    its = np.zeros(3, np.int32)
    rr = np.zeros(3)
    code = N.lib().bp_solve_batch(batch.build(), N.ptr(rhs), N.ptr(x), 1e-12, 2, 0, N.ptr(its), N.ptr(rr))
    assert code == N.BP_ERR_NOT_CONVERGED
    assert list(its) == [2, 2, 2] and np.all(rr > 1e-12)
    batch.close()
    ctx.close()
