"""The tuner's choice on given measurements (no device): candidates outside
the energy tolerance (worst entry) and unsupported orders are skipped, the
least cost wins, ties go to the earlier candidate."""
import pytest

from beep3_b200.autotune import Trial, autotune, choose


def trial(tree, size, cost, energies, status="ok", nterms=9):
    return Trial(tree, size, nterms, cost_ms=cost, energies=list(energies), status=status)


def test_choose_least_cost_within_tolerance():
    ts = [trial("reference", 1500, 18.0, [-100.0, -50.0]),
          trial("reference", 700, 14.5, [-100.005, -50.001]),
          trial("device", 96, 13.0, [-100.0, -50.02]),          # second energy outside 1e-4
          trial("reference", 1500, float("nan"), [], status="unsupported", nterms=18)]
    best = choose(ts, [-100.0, -50.0], 1e-4)
    assert (best.tree, best.size) == ("reference", 700)
    assert ts[2].status == "energy" and ts[3].status == "unsupported"
    assert best.settings() == dict(tree="reference", nbsize=700, nterms=9)


def test_choose_ties_and_no_candidate():
    ts = [trial("reference", 1000, 5.0, [-1.0]), trial("device", 64, 5.0, [-1.0])]
    assert choose(ts, [-1.0], 1e-4).size == 1000
    with pytest.raises(RuntimeError):
        choose([trial("device", 64, 1.0, [-2.0])], [-1.0], 1e-4)


def test_autotune_drives_the_trial():
    costs = {("reference", 1500): 10.0, ("reference", 700): 7.0, ("device", 96): 6.0}
    energy = {("reference", 1500): -10.0, ("reference", 700): -10.0005, ("device", 96): -10.01}
    seen = []

    def run(tree, size, nterms):
        seen.append((tree, size, nterms))
        if nterms != 9:
            return Trial(tree, size, nterms, status="unsupported")
        return Trial(tree, size, nterms, cost_ms=costs[(tree, size)], energies=[energy[(tree, size)]])

    res = autotune(run, candidates=tuple(costs), orders=(9, 18))
    assert len(seen) == 6
    assert res.settings() == dict(tree="reference", nbsize=700, nterms=9)
    assert res.reference_energies == [-10.0]
    assert [t.status for t in res.trials] == ["ok", "ok", "energy"] + ["unsupported"] * 3


def test_autotune_tries_compact_storage():
    """With compact=(False, True) every tree is tried with both near-field
    storages; the energy reference is the first FP32-coefficient candidate,
    and a cheaper compact candidate within the tolerance wins."""
    seen = []

    def run(tree, size, nterms, compact=False):
        seen.append((tree, size, compact))
        cost = {1500: 10.0, 700: 8.0}[size] - (1.5 if compact else 0.0)
        e = -10.0 - (2e-6 if compact else 0.0) - (1e-5 if size == 700 else 0.0)
        return Trial(tree, size, nterms, cost_ms=cost, energies=[e], compact=compact)

    res = autotune(run, candidates=(("reference", 1500), ("reference", 700)), compact=(False, True))
    assert seen == [("reference", 1500, False), ("reference", 700, False),
                    ("reference", 1500, True), ("reference", 700, True)]
    assert res.reference_energies == [-10.0]
    assert res.settings() == dict(tree="reference", nbsize=700, nterms=9, compact_nearfield=True)
    assert not res.trials[0].compact and res.trials[3].compact


def test_compact_is_unsupported_outside_the_mixed_engine():
    from beep3_b200.autotune import problem_trial

    def make(**kw):
        import beep3_b200 as b
        return b.BEEP(precision="fp64", **kw)

    t = problem_trial(make)("reference", 1500, 9, compact=True)
    assert t.status == "unsupported" and t.compact
