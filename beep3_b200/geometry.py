"""Surfaces, charges and node-patch preparation.

* :func:`icosphere` -- icosahedron subdivided ``k`` times (10*4^k + 2 vertices).
* :func:`star_surface` -- star-shaped molecule r(theta, phi) = R (1 + amp *
  sum_{l=1..lmax, m} a_lm Y_lm) with a_lm ~ N(0, 1)/(l + 1)^2 from a seed,
  on an icosphere's directions.
* :func:`charges_in_sphere`, :func:`charges_in_star` -- uniform point charges.
* :func:`prepare_patches` -- vertex-centred node patches and their point
  lists through the C ABI (planar or PN-curved triangles, the reference's
  constant-basis quadrature).
* :func:`quaternion_matrix`, :func:`random_quaternion` -- poses, with the
  reference's quaternion convention (src/common/math_vector.h:514-533).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace
from math import factorial

import numpy as np

from . import _native as N


# --------------------------------------------------------------------------- surfaces
def icosphere(k: int, radius: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """Vertices (V, 3) and anticlockwise (outward) triangles (T, 3)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(p, float) / np.linalg.norm(p) for p in verts]
    f = list(faces)
    for _ in range(k):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    V = np.array(v) * radius
    T = np.array(f, dtype=np.int32)
    # orient outward
    c = V[T].mean(axis=1)
    n = np.cross(V[T[:, 1]] - V[T[:, 0]], V[T[:, 2]] - V[T[:, 0]])
    flip = (n * c).sum(axis=1) < 0
    T[flip] = T[flip][:, [0, 2, 1]]
    return V, T


def real_sph_harm(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Orthonormal real spherical harmonic Y_lm (polar angle theta)."""
    am = abs(m)
    x = np.cos(theta)
    # associated Legendre P_l^am(x) without the Condon-Shortley phase
    pmm = np.ones_like(x)
    if am > 0:
        s = np.sqrt(np.maximum(0.0, 1 - x * x))
        fact = 1.0
        for _ in range(am):
            pmm = pmm * fact * s
            fact += 2.0
    if l == am:
        plm = pmm
    else:
        pmmp1 = x * (2 * am + 1) * pmm
        if l == am + 1:
            plm = pmmp1
        else:
            for ll in range(am + 2, l + 1):
                pll = ((2 * ll - 1) * x * pmmp1 - (ll + am - 1) * pmm) / (ll - am)
                pmm, pmmp1 = pmmp1, pll
            plm = pmmp1
    norm = np.sqrt((2 * l + 1) / (4 * np.pi) * factorial(l - am) / factorial(l + am))
    if m > 0:
        return np.sqrt(2) * norm * plm * np.cos(m * phi)
    if m < 0:
        return np.sqrt(2) * norm * plm * np.sin(am * phi)
    return norm * plm


@dataclass
class StarShape:
    radius: float
    amp: float
    coeffs: dict  # (l, m) -> a_lm

    def r_of(self, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
        s = np.zeros_like(theta)
        for (l, m), a in self.coeffs.items():
            s = s + a * real_sph_harm(l, m, theta, phi)
        return self.radius * (1.0 + self.amp * s)


def star_shape(radius: float, seed: int, lmax: int = 6, amp: float = 0.15) -> StarShape:
    rng = np.random.default_rng(seed)
    coeffs = {}
    for l in range(1, lmax + 1):
        for m in range(-l, l + 1):
            coeffs[(l, m)] = rng.standard_normal() / (l + 1) ** 2
    return StarShape(radius, amp, coeffs)


def star_surface(k: int, radius: float, seed: int, lmax: int = 6, amp: float = 0.15):
    """Star-shaped closed surface on an icosphere of subdivision k."""
    U, T = icosphere(k, 1.0)
    shape = star_shape(radius, seed, lmax, amp)
    theta = np.arccos(np.clip(U[:, 2], -1, 1))
    phi = np.arctan2(U[:, 1], U[:, 0])
    r = shape.r_of(theta, phi)
    if np.any(r <= 0):
        raise ValueError("star surface amplitude too large: non-positive radius")
    return U * r[:, None], T, shape


def charges_in_sphere(n: int, radius: float, seed: int, qmin: float = -1.0, qmax: float = 1.0) -> np.ndarray:
    """[n][4] x y z q, positions uniform in the ball, charges uniform."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        p = rng.uniform(-radius, radius, size=3)
        if p @ p < radius * radius:
            out.append(p)
    pos = np.array(out)
    q = rng.uniform(qmin, qmax, size=n)
    return np.ascontiguousarray(np.column_stack([pos, q]))


def charges_in_star(n: int, shape: StarShape, seed: int, frac: float = 0.8) -> np.ndarray:
    """[n][4] charges uniform in r < frac * r(theta, phi), q ~ U[-1, 1]."""
    rng = np.random.default_rng(seed)
    rmax = frac * shape.radius * (1 + shape.amp * 4.0)
    pos = np.zeros((0, 3))
    while len(pos) < n:
        p = rng.uniform(-rmax, rmax, size=(4 * n, 3))
        r = np.linalg.norm(p, axis=1)
        theta = np.arccos(np.clip(p[:, 2] / np.maximum(r, 1e-300), -1, 1))
        phi = np.arctan2(p[:, 1], p[:, 0])
        keep = r < frac * shape.r_of(theta, phi)
        pos = np.vstack([pos, p[keep]])
    pos = pos[:n]
    q = rng.uniform(-1.0, 1.0, size=n)
    return np.ascontiguousarray(np.column_stack([pos, q]))


# --------------------------------------------------------------------------- poses
def quaternion_matrix(q) -> np.ndarray:
    """Rotation matrix of the unit quaternion (a, b, c, d), a the scalar part."""
    a, b, c, d = (float(v) for v in q)
    return np.array([
        [1 + 2 * (-c * c - d * d), 2 * (b * c - a * d), 2 * (a * c + b * d)],
        [2 * (a * d + b * c), 1 + 2 * (-b * b - d * d), 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (a * b + c * d), 1 + 2 * (-b * b - c * c)],
    ])


def random_quaternion(rng: np.random.Generator) -> np.ndarray:
    """Uniformly distributed unit quaternion (Shoemake's method)."""
    u1, u2, u3 = rng.uniform(size=3)
    return np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                     np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)])[[3, 0, 1, 2]]


# --------------------------------------------------------------------------- patches
@dataclass
class PatchSet:
    """Node patches with their point lists (points are x y z nx ny nz w)."""

    centroid: np.ndarray
    normal: np.ndarray
    area: np.ndarray
    node: np.ndarray
    qual_off: np.ndarray
    qual: np.ndarray
    quad_off: np.ndarray
    quad: np.ndarray
    gal_off: np.ndarray
    gal: np.ndarray
    total_area: float
    planar_area: float

    @property
    def n(self) -> int:
        return len(self.area)

    def transformed(self, rot: np.ndarray, centre_old: np.ndarray, centre_new: np.ndarray) -> "PatchSet":
        """Rigid move p -> R (p - centre_old) + centre_new, n -> R n."""
        R = np.asarray(rot, float)

        def mv(p):
            return np.ascontiguousarray((p - centre_old) @ R.T + centre_new)

        def pts(a):
            b = a.copy()
            b[:, 0:3] = mv(a[:, 0:3])
            b[:, 3:6] = a[:, 3:6] @ R.T
            return np.ascontiguousarray(b)

        return replace(self, centroid=mv(self.centroid), normal=np.ascontiguousarray(self.normal @ R.T),
                       node=mv(self.node), qual=pts(self.qual), quad=pts(self.quad), gal=pts(self.gal))


def prepare_patches(vertices: np.ndarray, triangles: np.ndarray, planar: bool = False, qual_rule: int = 4,
                    quad_rule: int = 0, vertex_normals: np.ndarray | None = None) -> PatchSet:
    L = N.lib()
    V = np.ascontiguousarray(vertices, dtype=np.float64)
    T = np.ascontiguousarray(triangles, dtype=np.int32)
    VN = None if vertex_normals is None else np.ascontiguousarray(vertex_normals, dtype=np.float64)
    h = C.c_void_p()
    N.check(L.bp_geom_create(len(V), N.ptr(V), N.ptr(VN), len(T), N.ptr(T), int(planar), qual_rule, quad_rule,
                             C.byref(h)))
    try:
        n, nq, np_, ng = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        N.check(L.bp_geom_sizes(h, C.byref(n), C.byref(nq), C.byref(np_), C.byref(ng)))
        n = n.value
        out = dict(centroid=np.zeros((n, 3)), normal=np.zeros((n, 3)), area=np.zeros(n), node=np.zeros((n, 3)),
                   qual_off=np.zeros(n + 1, np.int32), qual=np.zeros((nq.value, 7)),
                   quad_off=np.zeros(n + 1, np.int32), quad=np.zeros((np_.value, 7)),
                   gal_off=np.zeros(n + 1, np.int32), gal=np.zeros((ng.value, 7)))
        totals = np.zeros(2)
        N.check(L.bp_geom_copy(h, *(N.ptr(out[k]) for k in ("centroid", "normal", "area", "node", "qual_off", "qual",
                                                              "quad_off", "quad", "gal_off", "gal")), N.ptr(totals)))
    finally:
        L.bp_geom_destroy(h)
    return PatchSet(**out, total_area=float(totals[0]), planar_area=float(totals[1]))
