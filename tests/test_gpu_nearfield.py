"""GPU parity of the near-field matvec, GMRES, right-hand side and energy
against the oracle, through the C ABI (Kirkwood sphere: the reference tree
does not subdivide 642 patches at nbsize 1500, so its matvec is the dense
near field)."""
import ctypes as C

import numpy as np
import pytest

import beep3_b200 as b
import oracle as O
from beep3_b200 import _native as N
from conftest import make_beep, rel_l2
from oracle import kirkwood as K

pytestmark = pytest.mark.gpu

# tolerances: FP64 path vs the FP64 oracle (same formulas, different
# summation order); mixed path (FP32 near field) vs the reference-faithful
# FP32 oracle at the parity bars (1e-5 on f/h, 1e-4 on energy)
TOL_FP64 = 1e-10
TOL_MIXED = 1e-5


@pytest.fixture(scope="module", params=["fp64", "mixed"])
def setup(request, kirkwood_case):
    prec = request.param
    bp = make_beep(kirkwood_case["mesh"], kappa=0.1, precision=prec)
    bp.build()
    arr = bp.gathered()
    pr = O.Problem(arr, bp.tree(), 0.1, fp32=(prec == "mixed"))
    yield prec, bp, pr
    bp.close()


def test_matvec_parity(setup):
    prec, bp, pr = setup
    rng = np.random.default_rng(3)
    for _ in range(2):
        x = rng.standard_normal(2 * pr.n)
        y = bp.matvec(x)
        yo = pr.matvec(x)
        assert rel_l2(y, yo) < (TOL_FP64 if prec == "fp64" else TOL_MIXED)


def test_info_and_tree(setup):
    prec, bp, pr = setup
    inf = bp.info()
    assert inf.n_patches == 642 and inf.n_levels == 1 and inf.fmm_active == 0
    assert inf.n_nearfield_pairs == 642 * 642
    assert pr.n_records == 642 + 642 * 642


def test_rhs_parity(setup):
    """FP64 engine: the exact FP64 direct sum.  Mixed engine: FP32 terms
    summed in FP64, held to 1e-6 -- the reference's own right-hand side comes
    from a 6-figure FMM."""
    prec, bp, pr = setup
    rhs = bp.set_rhs()
    ro = O.rhs(pr.patches, bp.instances[0].charges, 80.0)
    assert rel_l2(rhs, ro) < (1e-12 if prec == "fp64" else 1e-6)


def test_solve_and_energy(setup, kirkwood_case):
    prec, bp, pr = setup
    info = bp.solve(1e-6, 100)
    assert info.converged
    xo, its_o, _ = pr.solve(bp.rhs, 1e-6, 100)
    assert rel_l2(bp.x, xo) < (1e-8 if prec == "fp64" else TOL_MIXED)
    e, per = bp.calculate_energies()
    inst = bp.instances[0]
    arr = bp.gathered()
    ecf, ech = O.energy_coefficients(arr["gal_off"], arr["gal"], arr["area"], inst.charges,
                                     inst.mesh.patches.total_area)
    eo = O.energy(xo[:pr.n], xo[pr.n:], ecf, ech, inst.dielectric_ratio)
    assert abs(e - eo) / abs(eo) < (1e-8 if prec == "fp64" else 1e-4)
    ek = K.solvation_energy(inst.charges, 10.0, 2.0, 80.0, 0.1, centre=inst.offset)
    assert abs(e - ek) / abs(ek) < 0.015


def test_restarted_gmres_converges(setup):
    prec, bp, pr = setup
    bp.set_rhs()
    x, its, rr, ok = bp.gmres(1e-8, 200, restart=5)
    assert ok and rr <= 1e-8
    r = bp.matvec(x) - bp.rhs
    assert np.linalg.norm(r) / np.linalg.norm(bp.rhs) < 1e-6


def test_warm_start_runs_the_residual_matvec(setup):
    """x0 = 0 starts from r = -b without a matvec; a nonzero x0 (the
    converged solution, host and device entry points) starts from A x0 - b
    and stops at once."""
    prec, bp, pr = setup
    bp.set_rhs()
    x, its, rr, ok = bp.gmres(1e-8, 200)
    assert ok and its > 2
    x2, its2, rr2, ok2 = bp.gmres(1e-8, 200, x0=x)
    assert ok2 and its2 <= 1
    assert rel_l2(x2, x) < 1e-6  # one correction step within the 1e-8 stop test
    import torch
    xd = torch.tensor(x, device="cuda")
    bd = torch.tensor(bp.rhs, device="cuda")
    it, r = C.c_int32(), C.c_double()
    N.check(N.lib().bp_solve_device(bp.build(), bd.data_ptr(), xd.data_ptr(), 1e-8, 200, 0, C.byref(it), C.byref(r)))
    assert it.value <= 1 and rel_l2(xd.cpu().numpy(), x) < 1e-6


def test_kappa_zero_and_planar(kirkwood_case):
    mesh = b.Mesh(kirkwood_case["V"], kirkwood_case["T"], kirkwood_case["charges"], planar=True)
    bp = make_beep(mesh, kappa=0.0)
    pr = O.Problem(bp.gathered(), bp.host_tree(), 0.0, fp32=False)
    x = np.random.default_rng(1).standard_normal(2 * pr.n)
    assert rel_l2(bp.matvec(x), pr.matvec(x)) < TOL_FP64
    bp.close()


def test_device_entry_points_and_errors(kirkwood_case):
    import torch
    bp = make_beep(kirkwood_case["mesh"])
    p = bp.build()
    L = N.lib()
    x = torch.randn(2 * 642, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    N.check(L.bp_matvec_device(p, x.data_ptr(), y.data_ptr()))
    N.check(L.bp_ctx_synchronize(bp.context()))
    y_host = bp.matvec(x.cpu().numpy())
    assert rel_l2(y.cpu().numpy(), y_host) < 1e-13
    assert L.bp_matvec_device(p, x.data_ptr(), x.data_ptr()) == N.BP_ERR_INVALID
    bp.close()


def test_budget_is_enforced(kirkwood_case):
    bp = make_beep(kirkwood_case["mesh"], hbm_budget_bytes=1 << 20)
    with pytest.raises(b.BudgetExceeded):
        bp.build()
    bp.close()


def test_gmres_loop_runs_as_one_graph(kirkwood_case):
    """The Arnoldi loop of a cycle runs as one CUDA graph with a device-side
    loop condition (no host round trip per step)."""
    bp = make_beep(kirkwood_case["mesh"], precision="mixed")
    assert bp.info().gmres_graph == 0
    info = bp.solve(1e-6, 100)
    assert info.converged and bp.info().gmres_graph == 1
    bp.close()
