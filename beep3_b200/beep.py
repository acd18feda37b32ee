"""Host-side mirror of libBEEP's solver API (src/beep/beep.h:198-278).

``Mesh`` is a library mesh (surface + charges), ``MeshInstance`` a rigid
placement of one, ``BEEP`` the scenario: it gathers the node patches of all
instances, computes the bounding cube, the right-hand side, the adaptive
tree and the cached near field, runs GMRES with the B200 matvec and
evaluates solvation energies.  All compute goes through the C ABI of
``libbeep3_b200.so``.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .geometry import PatchSet, prepare_patches, quaternion_matrix

BETA0 = 1e-10  # screening standing in for the Laplace channels (src/beep/beep.cpp:32)
DEFAULT_NBSIZE = 1500  # DEFAULT_BEM_NEIGHBOURHOOD_SIZE, CPU build (src/beep/beep.h:74)


def _export_tree(export_fn, handle, n_points: int) -> dict:
    nn, nl, nc = C.c_int32(), C.c_int32(), C.c_int64()
    N.check(export_fn(handle, C.byref(nn), C.byref(nl), C.byref(nc), None, None, None))
    info = np.zeros((nn.value, 18), np.int32)
    geom = np.zeros((nn.value, 4))
    contents = np.zeros(nc.value, np.int32)
    N.check(export_fn(handle, None, None, None, N.ptr(info), N.ptr(geom), N.ptr(contents)))
    return dict(n_levels=nl.value, info=info, geom=geom, contents=contents)


def build_tree(points: np.ndarray, centre, edge: float, nbsize: int) -> dict:
    """Host-only adaptive octree (bp_tree_create) as numpy arrays."""
    L = N.lib()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    cen = np.ascontiguousarray(centre, dtype=np.float64)
    h = C.c_void_p()
    N.check(L.bp_tree_create(len(pts), N.ptr(pts), N.ptr(cen), float(edge), int(nbsize), C.byref(h)))
    try:
        return _export_tree(L.bp_tree_export, h, len(pts))
    finally:
        L.bp_tree_destroy(h)


class Mesh:
    """A library mesh: node patches of a closed surface and its point charges."""

    def __init__(self, vertices, triangles, charges, planar: bool = False, qual_rule: int = 4, quad_rule: int = 0,
                 centre=None, vertex_normals=None):
        self.vertices = np.ascontiguousarray(vertices, float)
        self.triangles = np.ascontiguousarray(triangles, np.int32)
        self.planar, self.qual_rule, self.quad_rule = bool(planar), int(qual_rule), int(quad_rule)
        self.vertex_normals = None if vertex_normals is None else np.ascontiguousarray(vertex_normals, float)
        self.charges = np.ascontiguousarray(np.asarray(charges, float).reshape(-1, 4))
        self.patches: PatchSet = prepare_patches(self.vertices, self.triangles, planar, qual_rule, quad_rule,
                                                 vertex_normals)
        nz = self.charges[self.charges[:, 3] != 0]
        if centre is None:
            # Mesh::calculate_charges_centroid (src/bem/mesh.cpp:1654-1670)
            centre = nz[:, :3].mean(axis=0) if len(nz) else np.zeros(3)
        self.centre = np.asarray(centre, float)
        # Mesh::calculate_radius: max distance of a patch centroid from the centre
        self.radius = float(np.max(np.linalg.norm(self.patches.centroid - self.centre, axis=1)))
        self._energy_coef = None

    @property
    def n_patches(self) -> int:
        return self.patches.n


@dataclass
class MeshInstance:
    mesh: Mesh
    offset: np.ndarray
    rotation: np.ndarray  # quaternion (a, b, c, d)
    eps_protein: float
    eps_solvent: float
    charges: np.ndarray = field(init=False)

    def __post_init__(self):
        self.place(self.offset, self.rotation)

    def place(self, offset, rotation) -> None:
        """NodePatch / Charge change_coordinate_frame (src/bem/node_patch.cpp:369-456).
        The charges move at once; the patches (host copy) on first use, as
        the engine places its own copy on the device."""
        self.offset = np.asarray(offset, float)
        self.rotation = np.asarray(rotation, float)
        self.matrix = quaternion_matrix(self.rotation)
        self._patches = None
        ch = self.mesh.charges.copy()
        ch[:, :3] = (ch[:, :3] - self.mesh.centre) @ self.matrix.T + self.offset
        self.charges = np.ascontiguousarray(ch)

    @property
    def patches(self) -> PatchSet:
        if self._patches is None:
            self._patches = self.mesh.patches.transformed(self.matrix, self.mesh.centre, self.offset)
        return self._patches

    @property
    def n_patches(self) -> int:
        return self.mesh.patches.n

    @property
    def dielectric_ratio(self) -> float:
        return self.eps_solvent / self.eps_protein

    @property
    def radius(self) -> float:
        return self.mesh.radius


class EngineContext:
    """A device context (bp_ctx) with the meshes it holds on the device, for
    scenarios (BEEP objects) that run one after another on it: the later ones
    upload no mesh and reuse the device blocks of the earlier ones.  One
    thread at a time."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_meshes: int = 8,
                 device_geometry: bool = False):
        """``max_meshes``: device-resident meshes kept; beyond it the least
        recently used one not needed by the scenario being built goes.
        ``device_geometry``: a mesh's node patches and point lists are
        generated on the device from its surface (bp_mesh_create_from_surface,
        bit for bit the host preparation) instead of being uploaded."""
        self.device = int(device)
        self.max_meshes = int(max_meshes)
        self.device_geometry = bool(device_geometry)
        self._ctx = C.c_void_p()
        N.check(N.lib().bp_ctx_create(self.device, int(hbm_budget_bytes), C.byref(self._ctx)))
        # id(mesh) -> [mesh, handle, build in which it was last used]; holding
        # the mesh keeps its id from being reused while the entry exists
        self._meshes: dict[int, list] = {}
        self._build = 0

    def begin_build(self) -> None:
        """Marks the start of a scenario build (its meshes are not evicted)."""
        self._build += 1

    @property
    def handle(self) -> C.c_void_p:
        return self._ctx

    def mesh_handle(self, mesh: Mesh) -> C.c_void_p:
        """The mesh's patches (its own frame) on the device, uploaded on first
        use (bp_mesh_create)."""
        entry = self._meshes.get(id(mesh))
        if entry is None:
            stale = sorted((e[2], k) for k, e in self._meshes.items() if e[2] < self._build)
            while len(self._meshes) >= self.max_meshes and stale:
                N.lib().bp_mesh_destroy(self._meshes.pop(stale.pop(0)[1])[1])
            h = C.c_void_p()
            if self.device_geometry:
                vn = mesh.vertex_normals
                N.check(N.lib().bp_mesh_create_from_surface(
                    self._ctx, len(mesh.vertices), N.ptr(mesh.vertices), N.ptr(vn), len(mesh.triangles),
                    N.ptr(mesh.triangles), int(mesh.planar), mesh.qual_rule, mesh.quad_rule,
                    N.ptr(np.ascontiguousarray(mesh.centre)), C.byref(h), None))
            else:
                p = mesh.patches
                pp = N.bp_patches(p.n, N.ptr(p.centroid), N.ptr(p.normal), N.ptr(p.area), None, None,
                                  N.ptr(p.qual_off), N.ptr(p.qual), N.ptr(p.quad_off), N.ptr(p.quad),
                                  N.ptr(p.gal_off), N.ptr(p.gal))
                N.check(N.lib().bp_mesh_create(self._ctx, C.byref(pp), N.ptr(np.ascontiguousarray(mesh.centre)),
                                               C.byref(h)))
            entry = [mesh, h, self._build]
            self._meshes[id(mesh)] = entry
        entry[2] = self._build
        return entry[1]

    def memory(self) -> tuple[int, int]:
        """(bytes in live device buffers, bytes of released blocks kept for reuse)."""
        used, budget, cached = C.c_uint64(), C.c_uint64(), C.c_uint64()
        N.check(N.lib().bp_ctx_memory(self._ctx, C.byref(used), C.byref(budget)))
        N.check(N.lib().bp_ctx_cache(self._ctx, C.byref(cached), 0))
        return int(used.value), int(cached.value)

    def release_cache(self) -> None:
        N.check(N.lib().bp_ctx_cache(self._ctx, None, 1))

    def close(self) -> None:
        for e in self._meshes.values():
            N.lib().bp_mesh_destroy(e[1])
        self._meshes = {}
        if self._ctx:
            # refused (and the context kept) while a problem made on it is alive
            N.check(N.lib().bp_ctx_destroy(self._ctx))
            self._ctx = C.c_void_p()


@dataclass
class RunInfo:
    num_iterations: int
    rel_residual: float
    converged: bool
    time_total_ms: float
    time_rhs_ms: float
    time_tree_ms: float
    time_precalcs_ms: float
    time_gmres_ms: float
    num_patches: int
    num_explicits: int
    fmm_active: bool


class BEEP:
    """Scenario and solver (mirror of libBEEP's BEEP class)."""

    def __init__(self, eps_solvent: float = 80.0, kappa: float = 0.1, nbsize: int = DEFAULT_NBSIZE,
                 nterms: int = 9, precision: str = "fp64", device: int = 0, hbm_budget_bytes: int = 0,
                 context: EngineContext | None = None, nearfield_on_demand: bool = False,
                 tree: str = "reference", leaf_size: int = 64, compact_nearfield: bool = False,
                 cache_mesh_pairs: bool = False):
        """``context``: an EngineContext shared with scenarios run before or
        after this one (its device and budget apply); by default the scenario
        has its own.  ``nearfield_on_demand``: recompute the near field in
        every matvec instead of caching its coefficients (the reference's
        uncached GPU path): no coefficient memory, the assembly's cost per
        matvec.  ``tree``: "reference" (the reference's octree rules, driven
        by ``nbsize``) or "device" (built on the GPU from Morton codes, at
        most ``leaf_size`` patches per leaf; same neighbourhood rule, a
        different near/far split, so results agree to the FMM's accuracy).
        ``compact_nearfield`` (mixed precision only): cache each FP32
        near-field coefficient rounded to 24 bits, 12 bytes a pair instead of
        16 (relative error at most 2^-16 per coefficient; no reference
        counterpart).  ``cache_mesh_pairs`` (mixed precision): keep the
        near-field coefficients of each mesh's own close patch pairs with
        the mesh, computed once in its frame, and look them up in every
        later problem with that mesh and kappa (rigid moves leave them
        unchanged; a scan's poses then integrate only the rest)."""
        self.eps_solvent = float(eps_solvent)
        self.kappa = float(kappa)
        self.nbsize = int(nbsize)
        self.nterms = int(nterms)
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self.nearfield_on_demand = bool(nearfield_on_demand)
        self.compact_nearfield = bool(compact_nearfield)
        self.cache_mesh_pairs = bool(cache_mesh_pairs)
        if self.compact_nearfield and (precision != "mixed" or self.nearfield_on_demand):
            raise ValueError("compact_nearfield needs precision='mixed' and cached coefficients")
        if tree not in ("reference", "device"):
            raise ValueError("tree must be 'reference' or 'device'")
        self.tree_kind = tree
        self.leaf_size = int(leaf_size)
        if self.leaf_size <= 0:
            raise ValueError("leaf_size must be positive")
        self.instances: list[MeshInstance] = []
        self.device = int(device)
        self.hbm_budget_bytes = int(hbm_budget_bytes)
        self._engine = context
        self._own_engine = context is None
        # rigid-body scans: keep each mesh's own-charge potential across moves
        self.cache_own_potentials = False
        # round the bounding cube's edge up to the grid 2^(k/8), so that
        # scenarios of nearly the same extent (the poses of a scan) share the
        # far-field tables and operators their context keeps; the tree then
        # differs from the exact cube's, within the FMM's truncation error
        self.snap_cube_edge = False
        if context is not None:
            self.device = context.device
        self._problem = None
        self.bounding_cube = None
        self._manual_cube = False
        self.x = None
        self.rhs = None

    # ----------------------------------------------------------------- scenario
    def insert_mesh_instance(self, mesh: Mesh, offset=None, rotation=(1.0, 0.0, 0.0, 0.0),
                             eps_protein: float = 2.0) -> int:
        off = mesh.centre if offset is None else offset
        self.instances.append(MeshInstance(mesh, np.asarray(off, float), np.asarray(rotation, float),
                                           float(eps_protein), self.eps_solvent))
        self._invalidate()
        return len(self.instances) - 1

    def move_mesh_instance(self, idx: int, offset, rotation) -> None:
        self.instances[idx].place(offset, rotation)
        self._invalidate()

    def set_bounding_cube(self, centre, edge: float) -> None:
        self.bounding_cube = (np.asarray(centre, float), float(edge))
        self._manual_cube = True
        self._invalidate()

    def calculate_bounding_cube(self):
        """BEEP::calculate_bounding_cube (src/beep/beep.cpp:1652-1697)."""
        if self._manual_cube:
            return self.bounding_cube
        lo = np.full(3, 1e99)
        hi = np.full(3, -1e99)
        for inst in self.instances:
            r = inst.radius
            lo = np.minimum(lo, inst.offset - r)
            hi = np.maximum(hi, inst.offset + r)
        edge = float(np.max(hi - lo))
        if edge <= 0:
            raise ValueError("degenerate bounding cube")
        if self.snap_cube_edge:
            edge = float(2.0 ** (np.ceil(np.log2(edge) * 8.0) / 8.0))
        self.bounding_cube = ((hi + lo) / 2.0, edge)
        return self.bounding_cube

    def _invalidate(self) -> None:
        if self._problem is not None:
            N.lib().bp_problem_destroy(self._problem)
            self._problem = None

    def close(self) -> None:
        self._invalidate()
        if self._own_engine and self._engine is not None:
            self._engine.close()
            self._engine = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------------------- gathered arrays
    def _gather(self) -> dict:
        insts = self.instances
        if not insts:
            raise ValueError("no mesh instances")
        cat = lambda xs: np.ascontiguousarray(np.concatenate(xs))

        def offsets(key):
            offs, base = [np.zeros(1, np.int32)], 0
            for inst in insts:
                o = getattr(inst.patches, key)
                offs.append(o[1:] + base)
                base += int(o[-1])
            return cat(offs).astype(np.int32)

        d = dict(
            centroid=cat([i.patches.centroid for i in insts]), normal=cat([i.patches.normal for i in insts]),
            area=cat([i.patches.area for i in insts]),
            eps=cat([np.full(i.patches.n, i.dielectric_ratio) for i in insts]),
            gc=cat([np.full(i.patches.n, 0.5) for i in insts]),
            qual_off=offsets("qual_off"), qual=cat([i.patches.qual for i in insts]),
            quad_off=offsets("quad_off"), quad=cat([i.patches.quad for i in insts]),
            gal_off=offsets("gal_off"), gal=cat([i.patches.gal for i in insts]),
        )
        d["first"] = np.cumsum([0] + [i.patches.n for i in insts])
        return d

    @property
    def num_patches(self) -> int:
        return sum(i.n_patches for i in self.instances)

    def _mesh_handle(self, mesh: Mesh) -> C.c_void_p:
        return self.engine.mesh_handle(mesh)

    @property
    def engine(self) -> EngineContext:
        """The engine context (created on first use unless one was given)."""
        if self._engine is None:
            self._engine = EngineContext(self.device, self.hbm_budget_bytes)
        return self._engine

    def context(self) -> C.c_void_p:
        """The device context handle."""
        return self.engine.handle

    def gathered(self) -> dict:
        """All instances' patch arrays concatenated in patch order (host)."""
        return self._gather()

    def host_tree(self) -> dict:
        """The adaptive octree built on the host (no device needed)."""
        centre, edge = self.calculate_bounding_cube()
        cen = np.ascontiguousarray(np.concatenate([i.patches.centroid for i in self.instances]))
        return build_tree(cen, centre, edge, self.nbsize)

    def build(self):
        """Tree + singular integrals + cached near field on the device.  The
        instances' meshes stay on the device between builds; each instance
        is placed there by its rigid move (bp_problem_create_posed)."""
        if self._problem is not None:
            return self._problem
        if not self.instances:
            raise ValueError("no mesh instances")
        self.context()
        self._arrays = {"first": np.cumsum([0] + [i.n_patches for i in self.instances])}
        centre, edge = self.calculate_bounding_cube()
        insts = (N.bp_instance * len(self.instances))()
        self.engine.begin_build()
        for k, inst in enumerate(self.instances):
            insts[k].mesh = self._mesh_handle(inst.mesh)
            insts[k].rotation[:] = [float(v) for v in inst.matrix.ravel()]
            insts[k].offset[:] = [float(v) for v in inst.offset]
            insts[k].dielectric_ratio = inst.dielectric_ratio
        flags = ((N.BP_FLAG_NEARFIELD_ON_DEMAND if self.nearfield_on_demand else 0) |
                 (N.BP_FLAG_DEVICE_TREE if self.tree_kind == "device" else 0) |
                 (N.BP_FLAG_COMPACT_NEARFIELD if self.compact_nearfield else 0) |
                 (N.BP_FLAG_MESH_PAIR_CACHE if self.cache_mesh_pairs else 0))
        prm = N.bp_params(self.kappa, BETA0, (C.c_double * 3)(*centre), edge,
                          self.leaf_size if self.tree_kind == "device" else self.nbsize, self.nterms,
                          N.BP_PREC_FP64 if self.precision == "fp64" else N.BP_PREC_MIXED, flags)
        h = C.c_void_p()
        N.check(N.lib().bp_problem_create_posed(self.context(), insts, len(self.instances), C.byref(prm), C.byref(h)))
        self._problem = h
        return h

    def info(self) -> N.bp_problem_info:
        inf = N.bp_problem_info()
        N.check(N.lib().bp_problem_info_get(self.build(), C.byref(inf)))
        return inf

    def tree(self) -> dict:
        """The adaptive octree as numpy arrays (see bp_problem_tree)."""
        return _export_tree(N.lib().bp_problem_tree, self.build(), self.num_patches)

    # ----------------------------------------------------------------- hot path
    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x (BEEP::do_bem_fmm_iteration)."""
        p = self.build()
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.shape != (2 * self.num_patches,):
            raise ValueError("x must have 2N entries")
        y = np.empty_like(x)
        N.check(N.lib().bp_matvec(p, N.ptr(x), N.ptr(y)))
        return y

    def set_rhs(self) -> np.ndarray:
        """BEEP::set_rhs with a direct Coulomb sum over all instances' charges.
        With ``cache_own_potentials`` set, each instance's potential at its
        own patches is computed once per mesh and kept with it across rigid
        moves (bp_rhs_posed); only the other instances' charges are summed
        per call."""
        p = self.build()
        if not self.cache_own_potentials:
            ch = np.ascontiguousarray(np.concatenate([i.charges for i in self.instances]))
            ch = np.ascontiguousarray(ch[ch[:, 3] != 0])
            rhs = np.empty(2 * self.num_patches)
            N.check(N.lib().bp_rhs(p, N.ptr(ch), len(ch), self.eps_solvent, N.ptr(rhs)))
            self.rhs = rhs
            return rhs
        own = [np.ascontiguousarray(i.mesh.charges[i.mesh.charges[:, 3] != 0]) for i in self.instances]
        ptrs = (C.c_void_p * len(own))(*[a.ctypes.data for a in own])
        counts = (C.c_int32 * len(own))(*[len(a) for a in own])
        rhs = np.empty(2 * self.num_patches)
        N.check(N.lib().bp_rhs_posed(p, C.cast(ptrs, C.c_void_p), C.cast(counts, C.c_void_p), self.eps_solvent,
                                     N.ptr(rhs)))
        self.rhs = rhs
        return rhs

    def gmres(self, tol: float = 1e-6, max_iterations: int = 100, restart: int = 0, x0=None):
        p = self.build()
        x = np.zeros(2 * self.num_patches) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        its, rr = C.c_int32(), C.c_double()
        code = N.lib().bp_solve(p, N.ptr(self.rhs), N.ptr(x), tol, max_iterations, restart, C.byref(its),
                                C.byref(rr))
        converged = code == N.BP_OK
        if code not in (N.BP_OK, N.BP_ERR_NOT_CONVERGED):
            N.check(code)
        self.x = x
        return x, its.value, rr.value, converged

    def solve(self, gmres_stop_criteria: float = 1e-6, max_iterations: int = 100, restart: int = 0,
              x0=None) -> RunInfo:
        """BEEP::solve (src/beep/beep.cpp:417-512)."""
        t0 = time.perf_counter()
        self.build()
        inf = self.info()
        t1 = time.perf_counter()
        self.set_rhs()
        t2 = time.perf_counter()
        _, its, rr, ok = self.gmres(gmres_stop_criteria, max_iterations, restart, x0)
        t3 = time.perf_counter()
        return RunInfo(its, rr, ok, (t3 - t0) * 1e3, (t2 - t1) * 1e3, inf.tree_ms, inf.assemble_ms,
                       (t3 - t2) * 1e3, self.num_patches, int(inf.n_nearfield_pairs), bool(inf.fmm_active))

    # ----------------------------------------------------------------- energies
    def _energy_coefficients(self, idx: int):
        inst = self.instances[idx]
        mesh = inst.mesh
        if mesh._energy_coef is None:
            # rigid-motion invariant: computed once per library mesh
            p = self.build()
            first = int(self._arrays["first"][idx])
            n = inst.n_patches
            cf, chh = np.empty(n), np.empty(n)
            ch = np.ascontiguousarray(inst.charges[inst.charges[:, 3] != 0])
            N.check(N.lib().bp_energy_coefficients(p, first, n, N.ptr(ch), len(ch), mesh.patches.total_area,
                                                   N.ptr(cf), N.ptr(chh)))
            mesh._energy_coef = (cf, chh)
        return mesh._energy_coef

    def calculate_energies(self) -> tuple[float, list[float]]:
        """Per-instance solvation energies in kJ/mol and their sum
        (BEEP::calculate_energies, src/beep/beep.cpp:572-595)."""
        if self.x is None:
            raise RuntimeError("solve first")
        p = self.build()
        out = []
        for idx, inst in enumerate(self.instances):
            cf, chh = self._energy_coefficients(idx)
            e = C.c_double()
            first = int(self._arrays["first"][idx])
            N.check(N.lib().bp_energy(p, first, inst.n_patches, N.ptr(cf), N.ptr(chh), inst.dielectric_ratio,
                                      N.ptr(self.x), C.byref(e)))
            out.append(e.value)
        return float(sum(out)), out
