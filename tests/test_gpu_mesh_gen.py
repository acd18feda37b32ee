"""Node patches and point lists generated on the device from a surface
(bp_mesh_create_from_surface) against the host preparation (bp_geom_create):
both run the same PN / PNG1 surface code, the device side without fused
multiply-adds, so the point lists are bitwise equal; a problem posed from
either mesh gives bitwise the same matvec, and the areas agree."""
import ctypes as C

import numpy as np
import pytest

import beep3_b200 as b
from beep3_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind, planar, qual, quad", [
    ("sphere", False, 4, 0), ("star", False, 4, 0), ("star", True, 4, 0), ("star", False, 6, 1),
    ("sphere", False, 0, 4), ("star", False, 7, 0)])
def test_device_mesh_equals_host_mesh(kind, planar, qual, quad):
    if kind == "sphere":
        V, T = b.icosphere(3, 10.0)
        ch = b.charges_in_sphere(10, 7.0, seed=1)
    else:
        V, T, shape = b.star_surface(3, 15.0, seed=4)
        ch = b.charges_in_star(20, shape, seed=5)
    mesh = b.Mesh(V, T, ch, planar=planar, qual_rule=qual, quad_rule=quad)
    ys = []
    for dev_geom in (False, True):
        ctx = b.EngineContext(0, device_geometry=dev_geom)
        bp = b.BEEP(kappa=0.1, nbsize=300, precision="fp64", context=ctx)
        bp.insert_mesh_instance(mesh, offset=mesh.centre + np.array([1.0, -2.0, 0.5]), rotation=(0.8, 0.6, 0.0, 0.0))
        x = np.random.default_rng(3).standard_normal(2 * bp.num_patches)
        ys.append(bp.matvec(x))
        bp.close()
        ctx.close()
    assert np.array_equal(ys[0], ys[1])
    # areas of the surface against the host preparation
    L = N.lib()
    ctx = C.c_void_p()
    N.check(L.bp_ctx_create(0, 0, C.byref(ctx)))
    h, totals = C.c_void_p(), np.zeros(2)
    N.check(L.bp_mesh_create_from_surface(ctx, len(V), N.ptr(mesh.vertices), None, len(T), N.ptr(mesh.triangles),
                                          int(planar), qual, quad, N.ptr(np.ascontiguousarray(mesh.centre)),
                                          C.byref(h), N.ptr(totals)))
    assert totals[0] == mesh.patches.total_area
    N.check(L.bp_mesh_destroy(h))
    N.check(L.bp_ctx_destroy(ctx))


def test_device_mesh_rejects_bad_surfaces():
    L = N.lib()
    ctx = C.c_void_p()
    N.check(L.bp_ctx_create(0, 0, C.byref(ctx)))
    V, T = b.icosphere(1, 5.0)
    V = np.ascontiguousarray(V)
    open_T = np.ascontiguousarray(T[:-1], np.int32)  # one triangle short: not closed
    h = C.c_void_p()
    cen = np.zeros(3)
    assert L.bp_mesh_create_from_surface(ctx, len(V), N.ptr(V), None, len(open_T), N.ptr(open_T), 0, 4, 0,
                                         N.ptr(cen), C.byref(h), None) == N.BP_ERR_INVALID
    T32 = np.ascontiguousarray(T, np.int32)
    assert L.bp_mesh_create_from_surface(ctx, len(V), N.ptr(V), None, len(T32), N.ptr(T32), 0, 5, 0,
                                         N.ptr(cen), C.byref(h), None) == N.BP_ERR_INVALID
    N.check(L.bp_ctx_destroy(ctx))
