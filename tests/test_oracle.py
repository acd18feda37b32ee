"""The oracle (CPU restatement) pinned against analytic solutions and the
committed golden fixtures."""
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from oracle import kirkwood as K
from conftest import make_beep, rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_kirkwood_series_born_limit():
    ch = np.array([[0.0, 0.0, 0.0, 1.0]])
    for kappa in (0.0,):
        e = K.solvation_energy(ch, 10.0, 2.0, 80.0, kappa)
        assert abs(e - K.born_energy(1.0, 10.0, 2.0, 80.0)) < 1e-12 * abs(e)
    # salt screens more: energy more negative with kappa > 0
    assert K.solvation_energy(ch, 10.0, 2.0, 80.0, 0.1) < K.solvation_energy(ch, 10.0, 2.0, 80.0, 0.0)


def test_kirkwood_series_symmetry():
    rng = np.random.default_rng(0)
    ch = np.column_stack([rng.uniform(-3, 3, (5, 3)), rng.uniform(-1, 1, 5)])
    e1 = K.solvation_energy(ch, 8.0, 4.0, 80.0, 0.05)
    # a rigid rotation of the charges leaves the energy unchanged
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    ch2 = ch.copy()
    ch2[:, :3] = ch[:, :3] @ R.T
    e2 = K.solvation_energy(ch2, 8.0, 4.0, 80.0, 0.05)
    assert abs(e1 - e2) < 1e-10 * abs(e1)


def oracle_solve(case, kappa, fp32):
    bp = make_beep(case["mesh"], kappa=kappa)
    arr = bp.gathered()
    tree = bp.host_tree()
    pr = O.Problem(arr, tree, kappa, fp32)
    inst = bp.instances[0]
    rhs = O.rhs(pr.patches, inst.charges, 80.0)
    x, its, rr = pr.solve(rhs, 1e-6, 100)
    ecf, ech = O.energy_coefficients(arr["gal_off"], arr["gal"], arr["area"], inst.charges,
                                     case["mesh"].patches.total_area)
    n = pr.n
    return x, its, O.energy(x[:n], x[n:], ecf, ech, inst.dielectric_ratio), inst


@pytest.mark.parametrize("kappa", [0.1, 0.0])
def test_oracle_bem_matches_kirkwood(kirkwood_case, kappa):
    x, its, e, inst = oracle_solve(kirkwood_case, kappa, fp32=True)
    ek = K.solvation_energy(inst.charges, 10.0, 2.0, 80.0, kappa, centre=inst.offset)
    # BEM discretisation error of a 642-patch PN sphere
    assert abs(e - ek) / abs(ek) < 0.015, (e, ek)
    assert its < 40


def test_oracle_precision_modes_agree(kirkwood_case):
    x32, _, e32, _ = oracle_solve(kirkwood_case, 0.1, fp32=True)
    x64, _, e64, _ = oracle_solve(kirkwood_case, 0.1, fp32=False)
    assert rel_l2(x32, x64) < 1e-5
    assert abs(e32 - e64) / abs(e64) < 1e-5


def test_golden_fixtures(kirkwood_case):
    """Regression pin of the oracle on the Kirkwood sphere (fixtures made by
    tests/golden/make_golden.py)."""
    g = np.load(GOLDEN / "kirkwood_k3.npz")
    bp = make_beep(kirkwood_case["mesh"], kappa=float(g["kappa"]))
    # the committed fixture was made from the same seeded inputs
    np.testing.assert_allclose(bp.instances[0].charges, g["charges"], rtol=0, atol=0)
    arr = bp.gathered()
    pr = O.Problem(arr, bp.host_tree(), float(g["kappa"]), fp32=False)
    y = pr.matvec(g["x"])
    assert rel_l2(y, g["y"]) < 1e-12
    d = O.singular(pr.patches, float(g["kappa"]), fp32=False)
    np.testing.assert_allclose(d, g["singular"], rtol=1e-12, atol=1e-14)
    rhs = O.rhs(pr.patches, bp.instances[0].charges, 80.0)
    assert rel_l2(rhs, g["rhs"]) < 1e-13
    x, its, e, _ = oracle_solve(kirkwood_case, float(g["kappa"]), fp32=False)
    assert abs(e - float(g["energy"])) < 1e-9 * abs(float(g["energy"]))
    assert abs(float(g["energy"]) - float(g["kirkwood"])) / abs(float(g["kirkwood"])) < 0.015
