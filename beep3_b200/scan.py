"""Rigid-body scans: solvation interaction energies of two molecules over
many poses (the use case of BEEP's Python loop, tools/pybeep.py:352 ->
insert_mesh_instance / move_mesh_instance / solve / calculate_energies).

Each pose places molecule B relative to molecule A; its scenario (both
instances) is solved with GMRES on the device and

    E_int(pose) = E(A + B) - E(A alone) - E(B alone)

in kJ/mol, with E the BEM solvation energy summed over instances
(BEEP::calculate_energies).  Poses are independent: several workers run
concurrently, each on its own engine context and CUDA stream (the calls
release the GIL), so their kernels overlap on the GPU; a worker keeps both
meshes on the device and places B on the device for each of its poses.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from .batch import ScenarioBatch
from .beep import BEEP, DEFAULT_NBSIZE, EngineContext, Mesh
from .geometry import random_quaternion


@dataclass
class Pose:
    rotation: np.ndarray  # quaternion applied to molecule B
    offset: np.ndarray    # centre of B relative to the centre of A


@dataclass
class ScanResult:
    energies: list         # E_int per pose, kJ/mol
    complex_energies: list
    e_a: float
    e_b: float
    seconds: float
    iterations: list

    @property
    def poses_per_s(self) -> float:
        return len(self.energies) / self.seconds


def random_poses(n: int, seed: int, rmin: float = 45.0, rmax: float = 80.0) -> list[Pose]:
    """Uniform random orientation of B and a centre-to-centre separation
    uniform in [rmin, rmax] along a uniform random direction."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        q = random_quaternion(rng)
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        out.append(Pose(q, d * rng.uniform(rmin, rmax)))
    return out


def _tree_kw(nbsize):
    """BEEP tree keywords: an nbsize, or a dict of tree settings (autotune)."""
    return dict(nbsize) if isinstance(nbsize, dict) else dict(nbsize=nbsize)


def _solve_energy(instances, kappa, precision, nbsize, device, tol, max_it, context=None, snap=False):
    bp = BEEP(eps_solvent=80.0, kappa=kappa, precision=precision, device=device, context=context, **_tree_kw(nbsize))
    bp.snap_cube_edge = snap
    try:
        for mesh, off, q in instances:
            bp.insert_mesh_instance(mesh, offset=off, rotation=q, eps_protein=2.0)
        info = bp.solve(tol, max_it)
        e, _ = bp.calculate_energies()
        return e, info.num_iterations, np.array(bp.x, float)
    finally:
        bp.close()


def _pose_guess(guess, k=1):
    """The initial guess of k poses' complexes from the isolated molecules'
    solutions (xa, xb, na, nb): per pose A's patches then B's, f for all
    poses, then h.  Each molecule's solution in its own frame is unchanged
    by a rigid move, so it is the complex's solution up to the interaction."""
    xa, xb, na, nb = guess
    f = np.concatenate([xa[:na], xb[:nb]] * k)
    h = np.concatenate([xa[na:], xb[nb:]] * k)
    return np.concatenate([f, h])


def _scan_worker(mesh_a, mesh_b, poses, idx, kappa, precision, nbsize, device, tol, max_it, context=None,
                 isolated=(), snap=False, guess=None):
    """Poses idx on one engine context: the two meshes stay on the device and
    each pose only moves instance B (a new tree, near field and far-field
    set-up, then the solve).  The single-molecule problems in ``isolated``
    are solved first, on the same context.  Returns (pose results, their
    energies)."""
    bp = BEEP(eps_solvent=80.0, kappa=kappa, precision=precision, device=device, context=context, **_tree_kw(nbsize))
    bp.cache_own_potentials = True  # instance B only moves: its own potential, and A's, stay
    bp.snap_cube_edge = snap
    out = []
    try:
        iso = [_solve_energy(inst, kappa, precision, nbsize, device, tol, max_it, context=bp.engine, snap=snap)[0]
               for inst in isolated]
        if not idx:
            return out, iso
        ident = np.array([1.0, 0.0, 0.0, 0.0])
        ca = mesh_a.centre
        bp.insert_mesh_instance(mesh_a, offset=ca, rotation=ident, eps_protein=2.0)
        bp.insert_mesh_instance(mesh_b, offset=ca + poses[idx[0]].offset, rotation=poses[idx[0]].rotation,
                                eps_protein=2.0)
        for k in idx:
            bp.move_mesh_instance(1, ca + poses[k].offset, poses[k].rotation)
            info = bp.solve(tol, max_it, x0=None if guess is None else _pose_guess(guess))
            e, _ = bp.calculate_energies()
            out.append((k, e, info.num_iterations))
    finally:
        bp.close()
    return out, iso


def _batch_worker(mesh_a, mesh_b, poses, chunks, kappa, precision, nbsize, device, tol, max_it, context=None,
                  isolated=(), snap=False, guess=None):
    """Batches of poses on one engine context: each chunk of poses is one
    batch problem (every pose a scenario of A and B), solved with shared
    launches.  The single-molecule problems in ``isolated`` are solved
    first.  Returns (pose results, their energies)."""
    eng = context if context is not None else EngineContext(device)
    out = []
    try:
        iso = [_solve_energy(inst, kappa, precision, nbsize, device, tol, max_it, context=eng, snap=snap)[0]
               for inst in isolated]
        ident = np.array([1.0, 0.0, 0.0, 0.0])
        ca = mesh_a.centre
        for chunk in chunks:
            scen = []
            for k in chunk:
                bp = BEEP(eps_solvent=80.0, kappa=kappa, precision=precision, device=device, context=eng,
                          **_tree_kw(nbsize))
                bp.snap_cube_edge = snap
                bp.insert_mesh_instance(mesh_a, offset=ca, rotation=ident, eps_protein=2.0)
                bp.insert_mesh_instance(mesh_b, offset=ca + poses[k].offset, rotation=poses[k].rotation,
                                        eps_protein=2.0)
                scen.append(bp)
            batch = ScenarioBatch(scen, context=eng)
            try:
                info = batch.solve(tol, max_it, x0=None if guess is None else _pose_guess(guess, len(chunk)))
                es = batch.calculate_energies()
            finally:
                batch.close()
            out.extend((k, e, its) for k, (e, _), its in zip(chunk, es, info.iterations))
    finally:
        if context is None:
            eng.close()
    return out, iso


def rigid_body_scan(mesh_a: Mesh, mesh_b: Mesh, poses: list[Pose], kappa: float = 0.1, precision: str = "mixed",
                    nbsize: int | dict = DEFAULT_NBSIZE, workers: int = 4, device: int = 0, tol: float = 1e-6,
                    max_iterations: int = 100, contexts: list | None = None,
                    snap_cube_edges: bool = False, batch: int = 1, cache_pairs: bool = False,
                    warm_start: bool = False) -> ScanResult:
    """``nbsize``: the reference tree's nbsize, or a dict of BEEP tree keywords
    (``TuneResult.settings()`` of autotune).  ``contexts``: EngineContexts
    for the workers (at least ``workers``), kept
    by the caller across scans so that the meshes and device blocks stay on
    the device; by default each worker has its own for this scan.
    ``snap_cube_edges``: round each pose's bounding-cube edge up to a grid
    (BEEP.snap_cube_edge), so that poses of similar extent share the
    far-field tables and operators a context keeps instead of computing them
    per pose; energies then differ from the exact cube's by the FMM's
    truncation error.  ``batch`` > 1: poses are solved ``batch`` at a time
    as the scenarios of one batch problem (ScenarioBatch), sorted by
    separation so that a batch's common cube edge is close to each pose's
    own; a pose's energy then differs from its own problem's by the FMM's
    truncation error (its tree is built in the batch's cube).
    ``cache_pairs`` (mixed precision): each worker's meshes keep the
    near-field coefficients of their own close patch pairs
    (BEEP(cache_mesh_pairs=True)), so a pose integrates only the pairs the
    cache does not hold; energies agree with the uncached scan to FP32
    rounding.
    ``warm_start``: the two isolated molecules are solved first and every
    pose's GMRES starts from their solutions (about half the iterations of
    a start from zero).  The complex's solution then differs from a cold
    start's within the GMRES tolerance, which moves the complex energies by
    a few 1e-6 but the interaction energies, their small difference, by up
    to a few 1e-3 relative: tighten ``tol`` where those matter."""
    t0 = time.perf_counter()
    if cache_pairs:
        nbsize = dict(_tree_kw(nbsize), cache_mesh_pairs=True)
    ident = np.array([1.0, 0.0, 0.0, 0.0])
    ca = mesh_a.centre
    workers = max(1, min(workers, len(poses)))
    if contexts is not None and len(contexts) < workers:
        raise ValueError("fewer engine contexts than workers")
    guess = None
    if warm_start:  # the isolated molecules first, on the first worker's context
        ctx0 = contexts[0] if contexts else EngineContext(device)
        try:
            e_a, _, xa = _solve_energy([(mesh_a, ca, ident)], kappa, precision, nbsize, device, tol, max_iterations,
                                       context=ctx0, snap=snap_cube_edges)
            e_b, _, xb = _solve_energy([(mesh_b, mesh_b.centre, ident)], kappa, precision, nbsize, device, tol,
                                       max_iterations, context=ctx0, snap=snap_cube_edges)
        finally:
            if not contexts:
                ctx0.close()
        guess = (xa, xb, mesh_a.n_patches, mesh_b.n_patches)

    def isolated_for(nw):
        # otherwise the isolated molecules are solved by workers 0 and 1 (0
        # alone when it is the only one) on their contexts, before their poses
        iso = [[] for _ in range(nw)]
        if not warm_start:
            iso[0].append([(mesh_a, ca, ident)])
            iso[1 % nw].append([(mesh_b, mesh_b.centre, ident)])
        return iso

    isolated = isolated_for(workers)
    if batch > 1:
        order = sorted(range(len(poses)), key=lambda k: float(np.linalg.norm(poses[k].offset)))
        chunks = [order[c:c + batch] for c in range(0, len(order), batch)]
        workers = max(1, min(workers, len(chunks)))
        isolated = isolated_for(workers)
        with ThreadPoolExecutor(max_workers=workers) as ex:
            fw = [ex.submit(_batch_worker, mesh_a, mesh_b, poses, chunks[w::workers], kappa, precision, nbsize,
                            device, tol, max_iterations, contexts[w] if contexts else None, isolated[w],
                            snap_cube_edges, guess)
                  for w in range(workers)]
            outs = [f.result() for f in fw]
    else:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            fw = [ex.submit(_scan_worker, mesh_a, mesh_b, poses, list(range(w, len(poses), workers)), kappa,
                            precision, nbsize, device, tol, max_iterations, contexts[w] if contexts else None,
                            isolated[w], snap_cube_edges, guess)
                  for w in range(workers)]
            outs = [f.result() for f in fw]
    if not warm_start:
        e_a = outs[0][1][0]
        e_b = outs[1 % workers][1][-1]
    res = sorted(r for o in outs for r in o[0])
    dt = time.perf_counter() - t0
    ec = [r[1] for r in res]
    return ScanResult([e - e_a - e_b for e in ec], ec, e_a, e_b, dt, [r[2] for r in res])


def scan_trial(mesh_a: Mesh, mesh_b: Mesh, poses: list[Pose], kappa: float = 0.1, precision: str = "mixed",
               workers: int = 4, batch: int = 1, device: int = 0, contexts: list | None = None,
               snap_cube_edges: bool = False, tol: float = 1e-6, max_iterations: int = 100, repeats: int = 1):
    """An autotune trial (beep3_b200.autotune) that runs a short scan of
    ``poses`` in the given worker / batch configuration with each candidate
    tree: cost = the best of ``repeats`` scans' time per pose, energies = the
    poses' complex energies."""
    from ._native import BP_ERR_UNSUPPORTED, BeepError
    from .autotune import Trial

    def run(tree: str, size: int, nterms: int, compact: bool = False) -> Trial:
        t = Trial(tree, size, nterms, compact=compact)
        if compact and precision != "mixed":
            t.status = "unsupported"
            return t
        best = float("inf")
        for _ in range(repeats):
            try:
                res = rigid_body_scan(mesh_a, mesh_b, poses, kappa=kappa, precision=precision,
                                      nbsize=t.settings(), workers=workers, device=device, tol=tol,
                                      max_iterations=max_iterations, contexts=contexts,
                                      snap_cube_edges=snap_cube_edges, batch=batch)
            except BeepError as e:
                if e.code == BP_ERR_UNSUPPORTED:
                    t.status = "unsupported"
                    return t
                raise
            best = min(best, res.seconds / len(poses) * 1e3)
            t.energies = list(res.complex_energies)
        t.cost_ms = best
        return t
    return run
