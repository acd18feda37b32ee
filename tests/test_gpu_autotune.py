"""The tuner on the device: every candidate built and solved, order 18
reported unsupported, the chosen candidate the cheapest of those within
1e-4 of the reference tree's energy, and its settings usable as BEEP
keywords; the scan trial on a few poses."""
import pytest

import beep3_b200 as b
from beep3_b200.autotune import autotune, problem_trial, scenario_factory
from beep3_b200.scan import random_poses, scan_trial

pytestmark = pytest.mark.gpu


def test_autotune_problem():
    V, T, shape = b.star_surface(5, 20.0, seed=401)
    mesh = b.Mesh(V, T, b.charges_in_star(100, shape, seed=402))
    ctx = b.EngineContext(0)
    make = scenario_factory([(mesh, mesh.centre, (1.0, 0.0, 0.0, 0.0), 2.0)], ctx, kappa=0.1, precision="mixed")
    res = autotune(problem_trial(make, repeats=1), candidates=(("reference", 1500), ("reference", 700),
                                                                ("reference", 300), ("device", 64),
                                                                ("device", 128)), orders=(9, 18))
    ok = [t for t in res.trials if t.status == "ok"]
    assert all(t.status == "unsupported" for t in res.trials if t.nterms == 18)
    assert res.best in ok and res.best.cost_ms == min(t.cost_ms for t in ok)
    ref = res.reference_energies[0]
    for t in ok:
        assert abs(t.energies[0] - ref) <= 1e-4 * abs(ref)
    bp = make(**res.settings())
    bp.solve(1e-6, 100)
    e, _ = bp.calculate_energies()
    bp.close()
    assert abs(e - ref) <= 1e-4 * abs(ref)
    ctx.close()


def test_autotune_compact_storage():
    """Both near-field storages per tree: the compact candidates build,
    solve within 1e-4 of the FP32 reference tree's energy (they are within
    about 1e-6) and the chosen settings build a problem."""
    V, T, shape = b.star_surface(5, 20.0, seed=407)
    mesh = b.Mesh(V, T, b.charges_in_star(100, shape, seed=408))
    ctx = b.EngineContext(0)
    make = scenario_factory([(mesh, mesh.centre, (1.0, 0.0, 0.0, 0.0), 2.0)], ctx, kappa=0.1, precision="mixed")
    res = autotune(problem_trial(make, repeats=1), candidates=(("reference", 1500), ("reference", 700)),
                   compact=(False, True))
    assert [t.compact for t in res.trials] == [False, False, True, True]
    assert all(t.status == "ok" for t in res.trials)
    ref = res.reference_energies[0]
    assert abs(res.trials[2].energies[0] - res.trials[0].energies[0]) <= 1e-5 * abs(ref)
    bp = make(**res.settings())
    bp.solve(1e-6, 100)
    bp.close()
    ctx.close()


def test_autotune_scan():
    va, ta, sa = b.star_surface(4, 20.0, seed=403)
    vb, tb, sb = b.star_surface(3, 12.0, seed=404)
    ma = b.Mesh(va, ta, b.charges_in_star(40, sa, seed=405))
    mb = b.Mesh(vb, tb, b.charges_in_star(10, sb, seed=406))
    poses = random_poses(4, seed=407, rmin=30.0, rmax=45.0)
    res = autotune(scan_trial(ma, mb, poses, workers=2, batch=2),
                   candidates=(("reference", 300), ("reference", 150), ("device", 48)))
    ok = [t for t in res.trials if t.status == "ok"]
    assert res.best in ok and len(res.best.energies) == 4
