"""Measured choice of the tree (and FMM order) for a workload.

The reference exposes its tree through one parameter, nbsize (the target
mean neighbourhood size of BEEP::init_fmm_octree, src/beep/beep.cpp:1585-1641
and src/fmm/octree.h:867-986), and fixes the BEM FMM at order 9
(FMM_BEM_Octree<9,9,67>).  Which tree is fastest on this engine depends on
the workload: the cached near field costs 16-32 bytes per pair per matvec
plus its assembly once per problem, the far field a latency-bound pass per
level, and where several problems run at once (a scan's workers) the
device's total work counts, not one problem's latency.  So the tuner runs
the workload itself with each candidate: a trial returns the workload's
cost and its energies; candidates whose energies differ from the reference
tree's by more than ``energy_tol`` (relative, the worst entry) are
discarded, and the cheapest of the rest wins.  Two trials are provided:

* ``problem_trial``: one scenario built and solved; cost = set-up +
  solves_per_problem x solve (a problem solved for several right-hand
  sides);
* ``beep3_b200.scan.scan_trial``: a short rigid-body scan in the scan's own
  worker and batch configuration; cost = time per pose.

Order 18 is tried when asked and recorded as unsupported: the engine's
far-field kernels are laid out for order 9.  With ``compact=(False, True)``
every candidate tree is also tried with the compact near field
(BEEP(compact_nearfield=True): coefficients rounded to 24 bits, 12 bytes a
pair; mixed precision only, recorded as unsupported otherwise); the energy
check applies to it as to any other candidate, against the reference tree
with FP32 coefficients.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from . import _native as N
from .beep import BEEP, DEFAULT_NBSIZE, EngineContext

# (tree kind, nbsize or leaf cap)
DEFAULT_CANDIDATES = (("reference", DEFAULT_NBSIZE), ("reference", 1000), ("reference", 700), ("reference", 500),
                      ("device", 96), ("device", 128), ("device", 192))


@dataclass
class Trial:
    tree: str
    size: int
    nterms: int
    cost_ms: float = float("nan")
    energies: list = field(default_factory=list)  # the workload's energies (kJ/mol)
    status: str = "ok"  # ok / energy / unsupported
    detail: dict = field(default_factory=dict)
    compact: bool = False  # the compact near field

    def settings(self) -> dict:
        """Keyword arguments of BEEP for this candidate."""
        if self.tree == "device":
            kw = dict(tree="device", leaf_size=self.size, nterms=self.nterms)
        else:
            kw = dict(tree="reference", nbsize=self.size, nterms=self.nterms)
        if self.compact:
            kw["compact_nearfield"] = True
        return kw


@dataclass
class TuneResult:
    best: Trial
    trials: list = field(default_factory=list)
    reference_energies: list = field(default_factory=list)

    def settings(self) -> dict:
        return self.best.settings()


def choose(trials: list[Trial], reference_energies, energy_tol: float) -> Trial:
    """Marks the candidates outside the energy tolerance and returns the one
    of least cost among the rest (ties: the earlier candidate)."""
    ref = np.asarray(reference_energies, float)
    best = None
    for t in trials:
        if t.status != "ok":
            continue
        e = np.asarray(t.energies, float)
        if e.shape != ref.shape or np.any(np.abs(e - ref) > energy_tol * np.abs(ref)):
            t.status = "energy"
            continue
        if best is None or t.cost_ms < best.cost_ms:
            best = t
    if best is None:
        raise RuntimeError("no candidate met the energy tolerance")
    return best


def autotune(trial: Callable[..., Trial], candidates=DEFAULT_CANDIDATES, orders=(9,), energy_tol: float = 1e-4,
             compact=(False,)) -> TuneResult:
    """``trial(tree, size, nterms)`` runs the workload with one candidate
    (``trial(tree, size, nterms, compact=True)`` for the compact near
    field).  The first candidate that runs at order 9 with FP32 coefficients
    is the reference for the energy check (by default the reference's own
    tree at its default nbsize)."""
    trials = [trial(tree, size, nt, compact=True) if c else trial(tree, size, nt)
              for c in compact for nt in orders for tree, size in candidates]
    ref = next(t for t in trials if t.nterms == 9 and not t.compact and t.status == "ok")
    best = choose(trials, ref.energies, energy_tol)
    return TuneResult(best, trials, list(ref.energies))


def problem_trial(make: Callable[..., BEEP], solves_per_problem: float = 1.0, tol: float = 1e-6,
                  max_iterations: int = 100, repeats: int = 2) -> Callable[[str, int, int], Trial]:
    """A trial that builds the scenario (``make(**tree keywords)``, a BEEP
    with its instances inserted) ``repeats`` times and keeps the fastest
    set-up and solve: cost = set-up + solves_per_problem x solve."""
    def run(tree: str, size: int, nterms: int, compact: bool = False) -> Trial:
        t = Trial(tree, size, nterms, compact=compact)
        best_setup = best_solve = float("inf")
        for _ in range(repeats):
            try:
                bp = make(**t.settings())
            except ValueError:  # the compact near field outside the mixed engine
                t.status = "unsupported"
                return t
            try:
                inf = bp.info()
            except N.BeepError as e:
                bp.close()
                if e.code == N.BP_ERR_UNSUPPORTED:
                    t.status = "unsupported"
                    return t
                raise
            try:
                info = bp.solve(tol, max_iterations)
                e, _ = bp.calculate_energies()
            finally:
                bp.close()
            best_setup = min(best_setup, inf.setup_ms)
            best_solve = min(best_solve, info.time_rhs_ms + info.time_gmres_ms)
            t.energies = [e]
            t.detail = dict(iterations=info.num_iterations)
        t.detail.update(setup_ms=best_setup, solve_ms=best_solve)
        t.cost_ms = best_setup + solves_per_problem * best_solve
        return t
    return run


def scenario_factory(instances, context: EngineContext, **fixed) -> Callable[..., BEEP]:
    """A ``make`` for problem_trial from (mesh, offset, rotation, eps_protein)
    tuples and fixed BEEP keywords (kappa, precision, ...)."""
    def make(**kw) -> BEEP:
        bp = BEEP(context=context, **fixed, **kw)
        for mesh, off, rot, eps in instances:
            bp.insert_mesh_instance(mesh, offset=off, rotation=rot, eps_protein=eps)
        return bp
    return make
