"""ORACLE -- test infrastructure only.

CPU restatement of libBEEP's BEM matvec path (near field, singular
integrals, plane-wave FMM, GMRES, right-hand side, energies) used as the
checker in tests/, in ``__graft_entry__.smoke()`` and as the CPU baseline in
``bench.py``.  Nothing in the ``beep3_b200`` package imports it.

The C++ part is built by ``oracle/Makefile`` into ``oracle/_build/liboracle.so``
(:func:`build` runs make when the library is missing or stale).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_lib = None
_native = False


def _cpu_tag() -> str:
    """Identifies this host's CPU (model and instruction-set flags)."""
    import hashlib
    try:
        text = Path("/proc/cpuinfo").read_text()
    except OSError:
        text = ""
    keep = [ln for ln in text.splitlines() if ln.startswith(("model name", "flags"))][:2]
    return hashlib.sha1("\n".join(keep).encode()).hexdigest()[:12]


def native_lib_path() -> Path:
    return HERE / "_build" / f"native-{_cpu_tag()}" / "liboracle.so"


def build(native: bool = False) -> Path:
    """Builds the portable library, or with ``native`` the -march=native one
    for this host's CPU (the timed CPU baseline)."""
    out = native_lib_path() if native else LIB
    srcs = list(HERE.glob("*.cpp")) + list(HERE.glob("*.h")) + [HERE / "Makefile"]
    if not out.exists() or any(s.stat().st_mtime > out.stat().st_mtime for s in srcs):
        cmd = ["make", "-C", str(HERE)]
        if native:
            cmd += ["native", f"NATIVE_DIR={out.parent.relative_to(HERE)}"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)
    return out


REFERENCE = Path("/root/reference")
REF_LIB = HERE / "_ref" / "libref_pieces.so"


def build_ref() -> Path | None:
    """Builds oracle/_ref/libref_pieces.so (the reference's own RIBESL and
    interaction table) when the reference tree is present; returns the
    library path when it exists."""
    src = HERE / "ref_pieces.cpp"
    if (REFERENCE / "src" / "fmm" / "bessel_gamma.h").exists():
        if not REF_LIB.exists() or src.stat().st_mtime > REF_LIB.stat().st_mtime:
            res = subprocess.run(["make", "-C", str(HERE), "ref", f"REFERENCE={REFERENCE}"], capture_output=True,
                                 text=True)
            if res.returncode != 0:
                raise RuntimeError("reference pieces build failed:\n" + res.stdout + res.stderr)
    return REF_LIB if REF_LIB.exists() else None


def ref_lib() -> C.CDLL | None:
    """The reference's own compiled pieces, or None when they are not built."""
    path = build_ref()
    if path is None:
        return None
    L = C.CDLL(str(path))
    L.ref_ribesl.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p]
    L.ref_ribesl.restype = C.c_int
    L.ref_interaction_list.argtypes = [C.c_void_p]
    L.ref_interaction_list.restype = C.c_int
    return L


def use_native() -> None:
    """Makes lib() load the -march=native build (call before the first use)."""
    global _native
    if _lib is not None and not _native:
        raise RuntimeError("the portable oracle library is already loaded")
    _native = True


class OrPatches(C.Structure):
    _fields_ = [("n", C.c_int32)] + [(k, C.c_void_p) for k in (
        "centroid", "normal", "area", "eps", "gc", "qual_off", "qual", "quad_off", "quad", "gal_off", "gal")]


class OrTree(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("n_levels", C.c_int32), ("info", C.c_void_p), ("geom", C.c_void_p),
                ("neighbours", C.c_void_p), ("contents", C.c_void_p), ("n_contents", C.c_int64)]


MATVEC_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(str(build(native=_native)))
        P = C.c_void_p
        L.or_pair_coefficients.argtypes = [C.POINTER(OrPatches), C.c_int, P, P, C.c_double, C.c_int, P]
        L.or_singular.argtypes = [C.POINTER(OrPatches), C.c_double, C.c_int, P]
        L.or_near_create.argtypes = [C.POINTER(OrPatches), C.POINTER(OrTree), C.c_double, C.c_int]
        L.or_near_create.restype = P
        L.or_near_destroy.argtypes = [P]
        L.or_near_count.argtypes = [P]
        L.or_near_count.restype = C.c_int64
        L.or_near_apply.argtypes = [P, P, P]
        L.or_point_sums.argtypes = [C.c_int, P, P, P, C.c_int, C.c_double, P, P]
        L.or_gmres.argtypes = [MATVEC_FN, P, C.c_int, P, P, C.c_double, C.c_int, C.c_int,
                               C.POINTER(C.c_double)]
        L.or_gmres.restype = C.c_int
        if hasattr(L, "or_fmm_create"):
            L.or_fmm_create.argtypes = [C.POINTER(OrPatches), C.POINTER(OrTree), C.c_double, C.c_double,
                                        C.c_double, C.c_int]
            L.or_fmm_create.restype = P
            L.or_fmm_destroy.argtypes = [P]
            L.or_fmm_apply.argtypes = [P, P, P]
            L.or_fmm_direct.argtypes = [C.POINTER(OrPatches), C.c_double, C.c_double, C.c_int, P, P, P, P]
            L.or_interaction_list.argtypes = [P]
            L.or_interaction_list.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dtype=dt)


class Patches:
    """Holds contiguous copies of the gathered patch arrays for the oracle."""

    def __init__(self, a: dict):
        self.a = {k: _c(a[k], np.int32 if k.endswith("_off") else np.float64)
                  for k in ("centroid", "normal", "area", "eps", "gc", "qual_off", "qual", "quad_off", "quad",
                            "gal_off", "gal")}
        self.n = len(self.a["area"])
        self.s = OrPatches(self.n, *(_p(self.a[k]) for k in (
            "centroid", "normal", "area", "eps", "gc", "qual_off", "qual", "quad_off", "quad", "gal_off", "gal")))


def neighbours_from_info(info: np.ndarray) -> np.ndarray:
    """[n][27] same-level neighbour node ids (nb = 9(dz+1) + 3(dy+1) + dx+1)."""
    key = {(int(r[0]), int(r[1]), int(r[2]), int(r[3])): k for k, r in enumerate(info)}
    out = np.full((len(info), 27), -1, np.int32)
    for k, r in enumerate(info):
        L, x, y, z = (int(v) for v in r[:4])
        for nb in range(27):
            dz, dy, dx = nb // 9 - 1, (nb % 9) // 3 - 1, nb % 3 - 1
            out[k, nb] = key.get((L, x + dx, y + dy, z + dz), -1)
    return out


class Tree:
    def __init__(self, t: dict):
        self.info = _c(t["info"], np.int32)
        self.geom = _c(t["geom"])
        self.contents = _c(t["contents"], np.int32)
        self.neigh = neighbours_from_info(self.info)
        self.n_levels = int(t["n_levels"])
        self.s = OrTree(len(self.info), self.n_levels, _p(self.info), _p(self.geom), _p(self.neigh),
                        _p(self.contents), len(self.contents))


def pair_coefficients(patches: Patches, I, J, kappa: float, fp32: bool) -> np.ndarray:
    I = _c(I, np.int32)
    J = _c(J, np.int32)
    out = np.zeros((len(I), 4))
    lib().or_pair_coefficients(C.byref(patches.s), len(I), _p(I), _p(J), kappa, int(fp32), _p(out))
    return out


def singular(patches: Patches, kappa: float, fp32: bool) -> np.ndarray:
    out = np.zeros((patches.n, 4))
    lib().or_singular(C.byref(patches.s), kappa, int(fp32), _p(out))
    return out


def point_sums(off, pts, charges, scale: float):
    off = _c(off, np.int32)
    pts = _c(pts)
    ch = _c(charges)
    n = len(off) - 1
    a, b = np.zeros(n), np.zeros(n)
    lib().or_point_sums(n, _p(off), _p(pts), _p(ch), len(ch), scale, _p(a), _p(b))
    return a, b


def rhs(patches: Patches, charges, eps_solvent: float) -> np.ndarray:
    """BEEP::set_rhs restated with a direct sum (src/beep/beep.cpp:1124-1260)."""
    ch = np.asarray(charges, float)
    ch = ch[ch[:, 3] != 0]
    a, b = point_sums(patches.a["qual_off"], patches.a["qual"], ch, 1.0 / (4 * np.pi * eps_solvent))
    return np.concatenate([a, b])


def energy_coefficients(gal_off, gal, area, charges, total_area: float):
    """Mesh::init_energy_precalcs + renormalise_energy_precalcs (src/bem/mesh.cpp:730-925)."""
    ch = np.asarray(charges, float)
    ch = ch[ch[:, 3] != 0]
    ech, ecf = point_sums(gal_off, gal, ch, 1.0 / (4 * np.pi))
    total_f = -ecf.sum()
    gauss_error = ch[:, 3].sum() - total_f
    ecf = ecf - (np.asarray(area) / total_area) * gauss_error
    return ecf, ech


CONVERT_KJ_PER_MOL = 6.02214179e23 * 1.60217646e-19 ** 2 / (8.85418782e-12 * 1.0e-10 * 1000.0)


def energy(f, h, ecf, ech, eps_ratio: float) -> float:
    """Mesh::calculate_energy (src/bem/mesh.cpp:1373-1404), Kahan sum, kJ/mol."""
    s = comp = 0.0
    for fi, hi, cf, chh in zip(f, h, ecf, ech):
        frag = hi * eps_ratio * chh - fi * cf
        y = frag - comp
        t = s + y
        comp = (t - s) - y
        s = t
    return s * 0.5 * CONVERT_KJ_PER_MOL


def far_pairs(tree: dict, n: int, targets) -> tuple[np.ndarray, np.ndarray]:
    """(target, source) pairs outside each target leaf's 27-box neighbourhood
    (the complement of the cached near field, Octree::get_neighbourhood_contents,
    src/fmm/octree.h:618-650), grouped by target."""
    info, contents = tree["info"], tree["contents"]
    neigh = neighbours_from_info(info)
    leaf_of = np.full(n, -1)
    for k, r in enumerate(info):
        if r[4] & 2:
            leaf_of[contents[r[6]:r[6] + r[7]]] = k
    T, S = [], []
    for t in targets:
        near = np.zeros(n, bool)
        for m in neigh[leaf_of[t]]:
            if m >= 0:
                near[contents[info[m, 6]:info[m, 6] + info[m, 7]]] = True
        s = np.nonzero(~near)[0]
        T.append(np.full(len(s), t))
        S.append(s)
    return np.concatenate(T).astype(np.int32), np.concatenate(S).astype(np.int32)


def direct_far(arrays: dict, tree: dict, kappa: float, x, targets, beta0: float = 1e-10) -> np.ndarray:
    """The exact far field at the targets (2N vector, zero elsewhere): the
    12-channel sum over every far pair that the plane-wave FMM approximates
    (the method of src/fmm/test_fmm.cpp:181-214).  Targets must be distinct."""
    pt = Patches(arrays)
    T, S = far_pairs(tree, pt.n, targets)
    x = _c(x)
    y = np.zeros(2 * pt.n)
    lib().or_fmm_direct(C.byref(pt.s), kappa, beta0, len(T), _p(T), _p(S), _p(x), _p(y))
    return y


def exact_rows(arrays: dict, tree: dict, kappa: float, x, targets, beta0: float = 1e-10) -> np.ndarray:
    """FP64 direct-sum oracle of the matvec rows of the targets (2N vector,
    zero elsewhere): the same discretisation with every near-field pair
    integrated in FP64 (the singular diagonal included) and the far field
    summed directly instead of by the FMM."""
    pt = Patches(arrays)
    n = pt.n
    tg = np.asarray(targets, np.int64)
    info, contents = tree["info"], tree["contents"]
    neigh = neighbours_from_info(info)
    leaf_of = np.full(n, -1)
    for k, r in enumerate(info):
        if r[4] & 2:
            leaf_of[contents[r[6]:r[6] + r[7]]] = k
    I, J = [], []
    for t in tg:
        cols = [contents[info[m, 6]:info[m, 6] + info[m, 7]] for m in neigh[leaf_of[t]] if m >= 0]
        cols = np.concatenate(cols)
        cols = cols[cols != t]
        I.append(np.full(len(cols), t))
        J.append(cols)
    I = np.concatenate(I).astype(np.int32)
    J = np.concatenate(J).astype(np.int32)
    coef = pair_coefficients(pt, I, J, kappa, fp32=False)
    x = _c(x)
    y = direct_far(arrays, tree, kappa, x, tg, beta0)
    f, h = x[:n], x[n:]
    np.add.at(y, I, coef[:, 1] * f[J] - coef[:, 0] * h[J])
    np.add.at(y, n + I, coef[:, 3] * f[J] - coef[:, 2] * h[J])
    # singular self-patch terms with the geometric corrections, targets only
    sub = {k: np.asarray(arrays[k])[tg] for k in ("centroid", "normal", "area", "eps", "gc")}
    for key, pts in (("qual", "qual_off"), ("quad", "quad_off"), ("gal", "gal_off")):
        off = np.asarray(arrays[pts])
        pieces = [np.asarray(arrays[key])[off[t]:off[t + 1]] for t in tg]
        sub[pts] = np.concatenate([[0], np.cumsum([len(q) for q in pieces])]).astype(np.int32)
        sub[key] = np.concatenate(pieces)
    d = singular(Patches(sub), kappa, fp32=False)
    y[tg] += d[:, 1] * f[tg] - d[:, 0] * h[tg]
    y[n + tg] += d[:, 3] * f[tg] - d[:, 2] * h[tg]
    return y


def row_errors(y, ref, targets, n) -> tuple[float, float]:
    """Relative L2 error of the f rows and of the h rows over the targets."""
    t = np.asarray(targets)
    ef = np.linalg.norm(y[t] - ref[t]) / np.linalg.norm(ref[t])
    eh = np.linalg.norm(y[n + t] - ref[n + t]) / np.linalg.norm(ref[n + t])
    return float(ef), float(eh)


class Problem:
    """Restated BEEP matvec over a given tree: cached near field (+ FMM)."""

    def __init__(self, arrays: dict, tree: dict, kappa: float, fp32: bool, beta0: float = 1e-10,
                 cube_edge: float | None = None, nterms: int = 9, far_field: bool = True):
        self.patches = Patches(arrays)
        self.tree = Tree(tree)
        self.n = self.patches.n
        self.kappa = kappa
        L = lib()
        self._near = L.or_near_create(C.byref(self.patches.s), C.byref(self.tree.s), kappa, int(fp32))
        self._fmm = None
        if far_field and self.tree.n_levels - 1 >= 2:
            if not hasattr(L, "or_fmm_create"):
                raise RuntimeError("the oracle has no far field")
            self._fmm = L.or_fmm_create(C.byref(self.patches.s), C.byref(self.tree.s), kappa, beta0,
                                        float(cube_edge), nterms)

    @property
    def n_records(self) -> int:
        return int(lib().or_near_count(self._near))

    def near(self, x) -> np.ndarray:
        x = _c(x)
        y = np.zeros(2 * self.n)
        lib().or_near_apply(self._near, _p(x), _p(y))
        return y

    def far(self, x) -> np.ndarray:
        y = np.zeros(2 * self.n)
        if self._fmm is not None:
            x = _c(x)
            lib().or_fmm_apply(self._fmm, _p(x), _p(y))
        return y

    def matvec(self, x) -> np.ndarray:
        return self.near(x) + self.far(x)

    def solve(self, b, tol: float = 1e-6, max_iters: int = 100, restart: int = 0, x0=None):
        b = _c(b)
        x = np.zeros(2 * self.n) if x0 is None else _c(x0).copy()

        @MATVEC_FN
        def mv(_user, xp, yp):
            xv = np.ctypeslib.as_array(xp, shape=(2 * self.n,))
            yv = np.ctypeslib.as_array(yp, shape=(2 * self.n,))
            yv[:] = self.matvec(xv.copy())

        rr = C.c_double()
        its = lib().or_gmres(mv, None, 2 * self.n, _p(b), _p(x), tol, max_iters, restart, C.byref(rr))
        return x, its, rr.value

    def close(self):
        L = lib()
        if self._near:
            L.or_near_destroy(self._near)
            self._near = None
        if self._fmm:
            L.or_fmm_destroy(self._fmm)
            self._fmm = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
