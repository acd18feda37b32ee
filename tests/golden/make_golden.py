"""Generates tests/golden/*.npz with the oracle (run from the repository root:
``python tests/golden/make_golden.py``).  The fixtures pin the oracle's
near field, singular integrals, right-hand side and solved energy on the
Kirkwood sphere (icosphere k=3, radius 10, 10 seeded charges in r < 7,
eps 2/80, kappa 0.1), together with the analytic Kirkwood energy."""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import beep3_b200 as b  # noqa: E402
import oracle as O  # noqa: E402
from oracle import kirkwood as K  # noqa: E402
from conftest import make_beep  # noqa: E402


def main():
    V, T = b.icosphere(3, 10.0)
    ch = b.charges_in_sphere(10, 7.0, seed=1234)
    mesh = b.Mesh(V, T, ch)
    kappa = 0.1
    bp = make_beep(mesh, kappa=kappa)
    arr = bp.gathered()
    pr = O.Problem(arr, bp.host_tree(), kappa, fp32=False)
    x = np.random.default_rng(99).standard_normal(2 * pr.n)
    y = pr.matvec(x)
    inst = bp.instances[0]
    rhs = O.rhs(pr.patches, inst.charges, 80.0)
    sol, its, rr = pr.solve(rhs, 1e-6, 100)
    ecf, ech = O.energy_coefficients(arr["gal_off"], arr["gal"], arr["area"], inst.charges, mesh.patches.total_area)
    n = pr.n
    e = O.energy(sol[:n], sol[n:], ecf, ech, inst.dielectric_ratio)
    ek = K.solvation_energy(inst.charges, 10.0, 2.0, 80.0, kappa, centre=inst.offset)
    np.savez_compressed(Path(__file__).parent / "kirkwood_k3.npz", kappa=kappa, charges=inst.charges, x=x, y=y,
                        singular=O.singular(pr.patches, kappa, fp32=False), rhs=rhs, solution=sol, energy=e,
                        kirkwood=ek, iterations=its)
    print("energy", e, "kirkwood", ek, "iterations", its)


if __name__ == "__main__":
    main()
