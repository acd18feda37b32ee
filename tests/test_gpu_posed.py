"""Posed problems: instances of device-resident meshes placed on the device
(bp_problem_create_posed, the path BEEP.build takes) give the same operator
as the same patches transformed on the host and passed whole
(bp_problem_create)."""
import ctypes as C

import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200 import _native as N
from beep3_b200.beep import BETA0
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _host_problem(bp):
    g = bp.gathered()
    centre, edge = bp.calculate_bounding_cube()
    pp = N.bp_patches(len(g["area"]), N.ptr(g["centroid"]), N.ptr(g["normal"]), N.ptr(g["area"]), N.ptr(g["eps"]),
                      N.ptr(g["gc"]), N.ptr(g["qual_off"]), N.ptr(g["qual"]), N.ptr(g["quad_off"]), N.ptr(g["quad"]),
                      N.ptr(g["gal_off"]), N.ptr(g["gal"]))
    prm = N.bp_params(bp.kappa, BETA0, (C.c_double * 3)(*centre), edge, bp.nbsize, bp.nterms,
                      N.BP_PREC_FP64 if bp.precision == "fp64" else N.BP_PREC_MIXED, 0)
    h = C.c_void_p()
    N.check(N.lib().bp_problem_create(bp.context(), C.byref(pp), C.byref(prm), C.byref(h)))
    return h


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-6)])
def test_posed_equals_host_transformed(precision, tol):
    V, T, shape = b.star_surface(4, 15.0, seed=11)
    ma = b.Mesh(V, T, b.charges_in_star(40, shape, seed=12))
    V2, T2, shape2 = b.star_surface(3, 10.0, seed=13)
    mb = b.Mesh(V2, T2, b.charges_in_star(20, shape2, seed=14))
    q = b.random_quaternion(np.random.default_rng(15))
    bp = b.BEEP(kappa=0.1, nbsize=300, precision=precision)
    try:
        bp.insert_mesh_instance(ma)
        bp.insert_mesh_instance(mb, offset=ma.centre + np.array([30.0, 5.0, -3.0]), rotation=q, eps_protein=4.0)
        assert bp.info().fmm_active
        x = np.random.default_rng(16).standard_normal(2 * bp.num_patches)
        y_posed = bp.matvec(x)
        h = _host_problem(bp)
        try:
            y_host = np.empty_like(x)
            N.check(N.lib().bp_matvec(h, N.ptr(x), N.ptr(y_host)))
        finally:
            N.lib().bp_problem_destroy(h)
        assert rel_l2(y_posed, y_host) < tol
        # a second pose on the same context reuses the device-resident meshes
        bp.move_mesh_instance(1, ma.centre + np.array([-25.0, 12.0, 8.0]), q[[0, 2, 3, 1]])
        y2 = bp.matvec(x[: 2 * bp.num_patches])
        h = _host_problem(bp)
        try:
            y2h = np.empty_like(y2)
            N.check(N.lib().bp_matvec(h, N.ptr(x), N.ptr(y2h)))
        finally:
            N.lib().bp_problem_destroy(h)
        assert rel_l2(y2, y2h) < tol
        assert len(bp.engine._meshes) == 2
    finally:
        bp.close()


def test_posed_rejects_bad_instances():
    V, T, shape = b.star_surface(3, 10.0, seed=21)
    m = b.Mesh(V, T, b.charges_in_star(10, shape, seed=22))
    bp = b.BEEP(kappa=0.1, nbsize=300, precision="fp64")
    try:
        bp.insert_mesh_instance(m)
        bp.build()
        inst = (N.bp_instance * 1)()
        inst[0].mesh = bp._mesh_handle(m)
        inst[0].rotation[:] = [1, 0, 0, 0, 1, 0, 0, 0, 1]
        inst[0].offset[:] = [0, 0, 0]
        inst[0].dielectric_ratio = -1.0
        centre, edge = bp.calculate_bounding_cube()
        prm = N.bp_params(0.1, BETA0, (C.c_double * 3)(*centre), edge, 300, 9, N.BP_PREC_FP64, 0)
        h = C.c_void_p()
        assert N.lib().bp_problem_create_posed(bp.context(), inst, 1, C.byref(prm), C.byref(h)) == N.BP_ERR_INVALID
        inst[0].dielectric_ratio = 40.0
        inst[0].offset[:] = [float("nan"), 0, 0]
        assert N.lib().bp_problem_create_posed(bp.context(), inst, 1, C.byref(prm), C.byref(h)) == N.BP_ERR_INVALID
    finally:
        bp.close()


def test_shared_context_reuses_and_evicts_meshes():
    """Scenarios run in turn on one EngineContext: a mesh seen before is not
    uploaded again, at most max_meshes stay resident, and every scenario gives
    the result it gives on a context of its own."""
    meshes = []
    for s in range(3):
        V, T, shape = b.star_surface(3, 10.0 + 2 * s, seed=31 + s)
        meshes.append(b.Mesh(V, T, b.charges_in_star(10, shape, seed=41 + s)))
    ectx = b.EngineContext(0, max_meshes=2)
    try:
        for m in meshes + meshes[:1]:
            own = b.BEEP(kappa=0.1, nbsize=300, precision="mixed")
            shared = b.BEEP(kappa=0.1, nbsize=300, precision="mixed", context=ectx)
            try:
                for bp in (own, shared):
                    bp.insert_mesh_instance(m)
                    bp.solve(1e-6, 50)
                e_own, _ = own.calculate_energies()
                e_shared, _ = shared.calculate_energies()
                assert e_shared == e_own
            finally:
                own.close()
                shared.close()
            assert len(ectx._meshes) <= 2
            assert id(m) in ectx._meshes
        used, cached = ectx.memory()
        assert cached > 0  # the last problem's blocks are kept for the next one
        ectx.release_cache()
        assert ectx.memory()[1] == 0
    finally:
        ectx.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-6)])
def test_posed_rhs_equals_direct_sum(precision, tol):
    """bp_rhs_posed (own-charge potentials kept with the meshes) against
    bp_rhs over all charges placed in the problem's frame, before and after a
    move; the second pose reuses the cached own-charge potentials."""
    V, T, shape = b.star_surface(4, 15.0, seed=51)
    ma = b.Mesh(V, T, b.charges_in_star(60, shape, seed=52))
    V2, T2, shape2 = b.star_surface(3, 10.0, seed=53)
    mb = b.Mesh(V2, T2, b.charges_in_star(25, shape2, seed=54))
    q = b.random_quaternion(np.random.default_rng(55))
    bp = b.BEEP(kappa=0.1, nbsize=300, precision=precision)
    bp.cache_own_potentials = True
    try:
        bp.insert_mesh_instance(ma)
        bp.insert_mesh_instance(mb, offset=ma.centre + np.array([28.0, -4.0, 6.0]), rotation=q, eps_protein=4.0)
        for pose in range(2):
            if pose:
                bp.move_mesh_instance(1, ma.centre + np.array([-22.0, 15.0, 3.0]), q[[0, 3, 1, 2]])
            r_posed = bp.set_rhs().copy()
            ch = np.ascontiguousarray(np.concatenate([i.charges for i in bp.instances]))
            r_direct = np.empty_like(r_posed)
            N.check(N.lib().bp_rhs(bp.build(), N.ptr(ch), len(ch), bp.eps_solvent, N.ptr(r_direct)))
            assert rel_l2(r_posed, r_direct) < tol
            assert np.array_equal(bp.set_rhs(), r_posed)  # cached own-charge potentials: same values
    finally:
        bp.close()


def test_mesh_destroyed_before_its_problem():
    """bp_mesh_destroy while a posed problem built from the mesh is alive
    defers the deletion; the problem's posed right-hand side still reads the
    mesh, and destroying the problem then frees it."""
    V, T, shape = b.star_surface(3, 10.0, seed=61)
    m = b.Mesh(V, T, b.charges_in_star(15, shape, seed=62))
    ectx = b.EngineContext(0)
    try:
        bp = b.BEEP(kappa=0.1, nbsize=300, precision="fp64", context=ectx)
        bp.insert_mesh_instance(m)
        h_mesh = ectx.mesh_handle(m)
        prm_centre, edge = bp.calculate_bounding_cube()
        inst = (N.bp_instance * 1)()
        inst[0].mesh = h_mesh
        inst[0].rotation[:] = [1, 0, 0, 0, 1, 0, 0, 0, 1]
        inst[0].offset[:] = list(m.centre)
        inst[0].dielectric_ratio = 40.0
        prm = N.bp_params(0.1, BETA0, (C.c_double * 3)(*prm_centre), edge, 300, 9, N.BP_PREC_FP64, 0)
        h = C.c_void_p()
        N.check(N.lib().bp_problem_create_posed(ectx.handle, inst, 1, C.byref(prm), C.byref(h)))
        try:
            del ectx._meshes[id(m)]
            N.check(N.lib().bp_mesh_destroy(h_mesh))  # deferred: the problem holds the mesh
            own = np.ascontiguousarray(m.charges[m.charges[:, 3] != 0])
            ptrs = (C.c_void_p * 1)(own.ctypes.data)
            counts = (C.c_int32 * 1)(len(own))
            r_posed = np.empty(2 * m.patches.n)
            N.check(N.lib().bp_rhs_posed(h, C.cast(ptrs, C.c_void_p), C.cast(counts, C.c_void_p), 80.0,
                                         N.ptr(r_posed)))
            world = np.ascontiguousarray(m.charges[m.charges[:, 3] != 0])  # identity placement
            r_direct = np.empty_like(r_posed)
            N.check(N.lib().bp_rhs(h, N.ptr(world), len(world), 80.0, N.ptr(r_direct)))
            assert rel_l2(r_posed, r_direct) < 1e-13
        finally:
            N.check(N.lib().bp_problem_destroy(h))  # the last user: frees the mesh
        bp.close()
    finally:
        ectx.close()
