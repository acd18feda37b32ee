"""Serving loop: continuous batching of BEM solves on one GPU.

Requests (one molecule each: surface + charges + kappa) arrive over time.
A request is admitted as soon as a worker slot is free and its device
footprint fits in the server's HBM budget: the footprint measured on an
earlier request of the same size and settings (the engine context's live
device bytes once the problem is built and solved), or, for a size not seen
yet, an upper estimate as the first guess; admitted requests run
concurrently, each on its own engine context (own CUDA stream), so their
kernels overlap on the device while later requests wait in the queue.
Device state (tree, near-field coefficients, FMM expansions, Krylov basis)
stays resident for the lifetime of a request and is released at completion,
which frees budget for the next admission.  Each worker slot keeps one
engine context for the requests it runs in turn, so a molecule seen before
is not uploaded again and a request reuses the device blocks its slot's
previous request released (those blocks are returned to the driver when an
admission needs their room).  Latency is measured from arrival to
completion.

The engine's kernels are deterministic (no atomics in any reduction), so a
request's result does not depend on what else is running.
"""
from __future__ import annotations

import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from .beep import BEEP, DEFAULT_NBSIZE, EngineContext, Mesh


@dataclass
class SolveRequest:
    mesh: Mesh
    kappa: float
    eps_protein: float = 2.0
    eps_solvent: float = 80.0
    tol: float = 1e-6
    max_iterations: int = 100
    tag: object = None
    arrival: float = field(default_factory=time.perf_counter)


@dataclass
class SolveResult:
    tag: object
    energy_kj_per_mol: float
    iterations: int
    converged: bool
    n_patches: int
    device_bytes: int
    arrival: float
    start: float
    end: float

    @property
    def latency_ms(self) -> float:
        return (self.end - self.arrival) * 1e3

    @property
    def queue_ms(self) -> float:
        return (self.start - self.arrival) * 1e3


def estimate_device_bytes(n_patches: int, nbsize: int, precision: str) -> int:
    """Upper estimate of a request's footprint: near-field coefficients
    (pairs ~ n * nbsize), FMM expansions and plane waves, Krylov basis."""
    coef = 16 if precision == "mixed" else 32
    pairs = n_patches * min(nbsize, n_patches) * 1.3
    fmm = n_patches / 4 * 12 * 55 * 16 * 2 + n_patches / 4 * 6 * 12 * 67 * 16
    krylov = 2 * n_patches * 8 * 110
    points = n_patches * 48 * 7 * 8 * 3
    return int(pairs * coef + fmm + krylov + points + (64 << 20))


class BemServer:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 64 << 30, workers: int = 4,
                 precision: str = "mixed", nbsize: int = DEFAULT_NBSIZE, restart: int = 0, runner=None,
                 estimator=None, tree_for=None):
        """``runner(req, need) -> SolveResult`` and ``estimator(req) -> bytes``
        default to the engine solve and :func:`estimate_device_bytes`.
        ``tree_for(n_patches) -> dict`` gives the BEEP tree keywords of a
        request by its size (for example the device-built tree for the
        largest ones, whose set-up it halves); by default every request
        uses the reference tree at ``nbsize``."""
        self.runner = runner or self._engine_solve
        self.estimator = estimator or (lambda r: estimate_device_bytes(r.mesh.n_patches, self.nbsize,
                                                                       self.precision))
        self.device = device
        self.budget = int(hbm_budget_bytes)
        self.precision = precision
        self.nbsize = nbsize
        self.tree_for = tree_for or (lambda n: dict(nbsize=self.nbsize))
        self.restart = restart
        self._pending: "queue.Queue[tuple[SolveRequest, Future] | None]" = queue.Queue()
        self._lock = threading.Condition()
        self._in_use = 0
        self._slots = workers
        self._threads: list[threading.Thread] = []
        self._contexts: list[EngineContext] = []  # idle engine contexts of the slots
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._closed = False
        self.peak_in_use = 0
        # measured device bytes per (patches, precision, nbsize, kappa > 0)
        self.measured_bytes: dict[tuple, int] = {}
        self._dispatcher.start()

    # -------------------------------------------------------------- public
    def submit(self, req: SolveRequest) -> Future:
        fut: Future = Future()
        self._pending.put((req, fut))
        return fut

    def close(self) -> None:
        self._pending.put(None)
        self._dispatcher.join()
        for t in self._threads:
            t.join()
        for c in self._contexts:
            c.close()
        self._contexts = []

    def _key(self, req: SolveRequest) -> tuple:
        tree = tuple(sorted(self.tree_for(req.mesh.n_patches).items()))
        return (req.mesh.n_patches, self.precision, tree, req.kappa > 0)

    def footprint(self, req: SolveRequest) -> int:
        """Device bytes reserved for a request: the largest measured on an
        earlier request of the same key, else the estimator's guess."""
        with self._lock:
            m = self.measured_bytes.get(self._key(req))
        return int(m) if m is not None else int(self.estimator(req))

    # -------------------------------------------------------------- internals
    def _dispatch(self) -> None:
        while True:
            item = self._pending.get()
            if item is None:
                return
            req, fut = item
            need = min(self.footprint(req), self.budget)
            with self._lock:
                # FIFO admission: wait for a slot and for budget to free up
                while self._slots == 0 or self._in_use + need > self.budget:
                    self._lock.wait()
                self._slots -= 1
                self._in_use += need
                self.peak_in_use = max(self.peak_in_use, self._in_use)
                if self.runner == self._engine_solve:
                    # blocks the idle slots keep for reuse count against the budget
                    kept = sum(c.memory()[1] for c in self._contexts)
                    if self._in_use + kept > self.budget:
                        for c in self._contexts:
                            c.release_cache()
            t = threading.Thread(target=self._run, args=(req, fut, need), daemon=True)
            self._threads.append(t)
            t.start()

    def _engine_solve(self, req: SolveRequest, need: int) -> SolveResult:
        start = time.perf_counter()
        with self._lock:
            ectx = self._contexts.pop() if self._contexts else None
        if ectx is None:
            ectx = EngineContext(self.device)
        bp = BEEP(eps_solvent=req.eps_solvent, kappa=req.kappa, precision=self.precision, context=ectx,
                  **self.tree_for(req.mesh.n_patches))
        try:
            bp.insert_mesh_instance(req.mesh, eps_protein=req.eps_protein)
            info = bp.solve(req.tol, req.max_iterations, restart=self.restart)
            e, _ = bp.calculate_energies()
            dev_bytes = int(bp.info().device_bytes)
            return SolveResult(req.tag, e, info.num_iterations, info.converged, bp.num_patches, dev_bytes,
                               req.arrival, start, time.perf_counter())
        finally:
            bp.close()  # the problem; the context goes back to the idle slots
            with self._lock:
                self._contexts.append(ectx)

    def _run(self, req: SolveRequest, fut: Future, need: int) -> None:
        res = None
        try:
            res = self.runner(req, need)
        except BaseException as exc:  # reported through the future
            fut.set_exception(exc)
        finally:
            with self._lock:
                if res is not None and res.device_bytes > 0:
                    k = self._key(req)
                    self.measured_bytes[k] = max(self.measured_bytes.get(k, 0), int(res.device_bytes))
                self._slots += 1
                self._in_use -= need
                self._lock.notify_all()
        if res is not None:
            fut.set_result(res)


def latency_percentiles(results: list[SolveResult]) -> dict:
    lat = np.array([r.latency_ms for r in results])
    return {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
            "mean": float(lat.mean())}
