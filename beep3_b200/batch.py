"""Independent scenarios solved together: one batch problem
(bp_problem_create_batch) whose matvecs and GMRES steps cover every
scenario in the same kernel launches.

A scenario is a BEEP object with its mesh instances inserted (the
reference's BEEP::insert_mesh_instance / move_mesh_instance,
src/beep/beep.cpp:223-290); the batch solves each one as BEEP::solve and
BEEP::calculate_energies would (src/beep/beep.cpp:417-512, :572-595), with
its own tree, right-hand side, Krylov basis and stop test.  The scenarios'
trees share one cube edge (the largest of theirs), so they share the
far-field operators; each scenario's tree is the one its own problem builds
in a cube of that edge around its centre (BEEP.set_bounding_cube).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .beep import BEEP, BETA0, EngineContext


@dataclass
class BatchSolve:
    iterations: list       # GMRES iterations per scenario
    rel_residuals: list    # residual estimate / ||rhs|| per scenario
    converged: list
    time_ms: float         # right-hand side + GMRES of the whole batch
    time_rhs_ms: float
    time_gmres_ms: float


class ScenarioBatch:
    """``scenarios``: BEEP objects with the same kappa, precision, solvent
    permittivity, FMM order and tree settings; their instances are read when
    the batch is built.  ``context``: the engine context holding the meshes
    (shared with the caller's other batches); by default the batch has its
    own.  ``cube_edge``: the common cube edge (at least every scenario's
    own); by default the largest of the scenarios' cubes."""

    def __init__(self, scenarios: list[BEEP], context: EngineContext | None = None, cube_edge: float | None = None):
        if not scenarios:
            raise ValueError("no scenarios")
        s0 = scenarios[0]
        for s in scenarios:
            if not s.instances:
                raise ValueError("a scenario without mesh instances")
            same = (s.kappa == s0.kappa and s.precision == s0.precision and s.eps_solvent == s0.eps_solvent
                    and s.nterms == s0.nterms and s.tree_kind == s0.tree_kind and s.nbsize == s0.nbsize
                    and s.leaf_size == s0.leaf_size and s.nearfield_on_demand == s0.nearfield_on_demand
                    and s.compact_nearfield == s0.compact_nearfield and s.cache_mesh_pairs == s0.cache_mesh_pairs)
            if not same:
                raise ValueError("the scenarios of a batch need the same kappa, precision, solvent, order and tree")
        self.scenarios = list(scenarios)
        cubes = [s.calculate_bounding_cube() for s in scenarios]
        self.centres = np.array([c for c, _ in cubes], dtype=np.float64)
        edge = max(e for _, e in cubes)
        if cube_edge is not None:
            if cube_edge < edge:
                raise ValueError("cube_edge is smaller than a scenario's extent")
            edge = float(cube_edge)
        self.cube_edge = float(edge)
        self._engine = context
        self._own_engine = context is None
        self._problem = None
        self.x = None
        # instance i of the batch: (scenario, index in it, first patch)
        self._inst = []
        first = 0
        for k, s in enumerate(scenarios):
            for j, inst in enumerate(s.instances):
                self._inst.append((k, j, first))
                first += inst.n_patches
        self.num_patches = first
        self.scenario_first_patch = [0]
        for s in scenarios:
            self.scenario_first_patch.append(self.scenario_first_patch[-1] + sum(i.n_patches for i in s.instances))

    @property
    def engine(self) -> EngineContext:
        if self._engine is None:
            s0 = self.scenarios[0]
            self._engine = EngineContext(s0.device, s0.hbm_budget_bytes)
        return self._engine

    def build(self):
        """The batch problem on the device (built once)."""
        if self._problem is not None:
            return self._problem
        s0 = self.scenarios[0]
        eng = self.engine
        eng.begin_build()
        all_inst = [inst for s in self.scenarios for inst in s.instances]
        insts = (N.bp_instance * len(all_inst))()
        for k, inst in enumerate(all_inst):
            insts[k].mesh = eng.mesh_handle(inst.mesh)
            insts[k].rotation[:] = [float(v) for v in inst.matrix.ravel()]
            insts[k].offset[:] = [float(v) for v in inst.offset]
            insts[k].dielectric_ratio = inst.dielectric_ratio
        sfirst = np.zeros(len(self.scenarios) + 1, np.int32)
        for k, s in enumerate(self.scenarios):
            sfirst[k + 1] = sfirst[k] + len(s.instances)
        centres = np.ascontiguousarray(self.centres.ravel())
        flags = ((N.BP_FLAG_NEARFIELD_ON_DEMAND if s0.nearfield_on_demand else 0) |
                 (N.BP_FLAG_DEVICE_TREE if s0.tree_kind == "device" else 0) |
                 (N.BP_FLAG_COMPACT_NEARFIELD if s0.compact_nearfield else 0) |
                 (N.BP_FLAG_MESH_PAIR_CACHE if s0.cache_mesh_pairs else 0))
        prm = N.bp_params(s0.kappa, BETA0, (C.c_double * 3)(0.0, 0.0, 0.0), self.cube_edge,
                          s0.leaf_size if s0.tree_kind == "device" else s0.nbsize, s0.nterms,
                          N.BP_PREC_FP64 if s0.precision == "fp64" else N.BP_PREC_MIXED, flags)
        h = C.c_void_p()
        N.check(N.lib().bp_problem_create_batch(eng.handle, insts, len(all_inst), N.ptr(sfirst), len(self.scenarios),
                                                N.ptr(centres), C.byref(prm), C.byref(h)))
        self._problem = h
        return h

    def info(self) -> N.bp_problem_info:
        inf = N.bp_problem_info()
        N.check(N.lib().bp_problem_info_get(self.build(), C.byref(inf)))
        return inf

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x of every scenario (block diagonal), in the batch's patch
        order: [f of all scenarios' patches, h of all scenarios' patches]."""
        p = self.build()
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.shape != (2 * self.num_patches,):
            raise ValueError("x must have 2N entries")
        y = np.empty_like(x)
        N.check(N.lib().bp_matvec(p, N.ptr(x), N.ptr(y)))
        return y

    def scenario_part(self, v: np.ndarray, k: int) -> np.ndarray:
        """Scenario k's entries of a batch vector, as its own problem orders
        them ([f of its patches, h of its patches])."""
        a, b = self.scenario_first_patch[k], self.scenario_first_patch[k + 1]
        n = self.num_patches
        return np.concatenate([v[a:b], v[n + a:n + b]])

    def set_rhs(self) -> np.ndarray:
        """Every scenario's right-hand side (bp_rhs_posed: each instance's
        own-charge potential kept with its mesh, the other instances of its
        scenario summed)."""
        p = self.build()
        all_inst = [inst for s in self.scenarios for inst in s.instances]
        own = [np.ascontiguousarray(i.mesh.charges[i.mesh.charges[:, 3] != 0]) for i in all_inst]
        ptrs = (C.c_void_p * len(own))(*[a.ctypes.data for a in own])
        counts = (C.c_int32 * len(own))(*[len(a) for a in own])
        rhs = np.empty(2 * self.num_patches)
        N.check(N.lib().bp_rhs_posed(p, C.cast(ptrs, C.c_void_p), C.cast(counts, C.c_void_p),
                                     self.scenarios[0].eps_solvent, N.ptr(rhs)))
        self.rhs = rhs
        return rhs

    def solve(self, gmres_stop_criteria: float = 1e-6, max_iterations: int = 100, restart: int = 0,
              x0=None) -> BatchSolve:
        """Right-hand sides, then every scenario's GMRES in shared launches,
        from ``x0`` (the batch's f for all patches, then h) or from zero."""
        p = self.build()
        t0 = time.perf_counter()
        self.set_rhs()
        t1 = time.perf_counter()
        S = len(self.scenarios)
        x = np.zeros(2 * self.num_patches)
        if x0 is not None:
            x[:] = np.asarray(x0, float).reshape(-1)
        its = np.zeros(S, np.int32)
        rr = np.zeros(S)
        code = N.lib().bp_solve_batch(p, N.ptr(self.rhs), N.ptr(x), gmres_stop_criteria, max_iterations, restart,
                                      N.ptr(its), N.ptr(rr))
        if code not in (N.BP_OK, N.BP_ERR_NOT_CONVERGED):
            N.check(code)
        t2 = time.perf_counter()
        self.x = x
        return BatchSolve([int(v) for v in its], [float(v) for v in rr],
                          [bool(v <= gmres_stop_criteria) for v in rr], (t2 - t0) * 1e3, (t1 - t0) * 1e3,
                          (t2 - t1) * 1e3)

    def calculate_energies(self) -> list[tuple[float, list[float]]]:
        """Per scenario: its total solvation energy in kJ/mol and the
        per-instance energies (BEEP::calculate_energies)."""
        if self.x is None:
            raise RuntimeError("solve first")
        p = self.build()
        out = [(0.0, []) for _ in self.scenarios]
        for k, j, first in self._inst:
            inst = self.scenarios[k].instances[j]
            mesh = inst.mesh
            if mesh._energy_coef is None:  # rigid-motion invariant: once per library mesh
                n = inst.n_patches
                cf, chh = np.empty(n), np.empty(n)
                ch = np.ascontiguousarray(inst.charges[inst.charges[:, 3] != 0])
                N.check(N.lib().bp_energy_coefficients(p, first, n, N.ptr(ch), len(ch), mesh.patches.total_area,
                                                       N.ptr(cf), N.ptr(chh)))
                mesh._energy_coef = (cf, chh)
            cf, chh = mesh._energy_coef
            e = C.c_double()
            N.check(N.lib().bp_energy(p, first, inst.n_patches, N.ptr(cf), N.ptr(chh), inst.dielectric_ratio,
                                      N.ptr(self.x), C.byref(e)))
            out[k][1].append(e.value)
        return [(float(sum(es)), es) for _, es in out]

    def tree(self) -> dict:
        """The batch's forest of trees (one per scenario) as numpy arrays."""
        from .beep import _export_tree
        return _export_tree(N.lib().bp_problem_tree, self.build(), self.num_patches)

    def close(self) -> None:
        if self._problem is not None:
            N.lib().bp_problem_destroy(self._problem)
            self._problem = None
        if self._own_engine and self._engine is not None:
            self._engine.close()
            self._engine = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
