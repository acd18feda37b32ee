"""Benchmark of the BEM matvec / GMRES solve (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   # CPU restatement of the reference path

A step is one matvec y = A x of the whole problem (near field + FMM) with x
already in HBM; ``value`` is matvecs/s of the mixed-precision engine
(whole job: sum over ranks / max time).  ``e2e`` is the same through the
host-buffer C-ABI call (bp_matvec: H2D of x and D2H of y inside the timed
region).  Extra keys report the FP64 engine, full solves/s, solve latency
percentiles and the mixed-vs-FP64 energy error.  Multi-GPU runs are
independent replicas (the path does not shard): scaling "weak".
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "BEM matvec/s & solves/s, mixed vs FP64 at <=1e-4 energy err; p50/p99 latency"
L2_BYTES = 126 * 1024 * 1024


# --------------------------------------------------------------------------- workloads
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one near-field
# apply launch, measured with ncu on each workload (a one-pass capture of the
# same bench command; 976.9 MB of them are algorithmic on the star workload)
APPLY_TRAFFIC = {"star": 983_633_408}


def workload(name: str):
    """Returns (description dict, list of (Mesh, offset, quaternion), kappa, nbsize)."""
    import beep3_b200 as b
    if name == "kirkwood":
        V, T = b.icosphere(3, 10.0)
        mesh = b.Mesh(V, T, b.charges_in_sphere(10, 7.0, seed=1234))
        desc = dict(workload="kirkwood sphere r=10 A, icosphere k=3 (642 patches), 10 charges, eps 2/80, "
                             "kappa 0.1, qual 4 / quad 0, reference tree nbsize 1500", patches=642)
        return desc, [(mesh, None, (1, 0, 0, 0))], 0.1, 1500
    if name == "star":
        V, T, shape = b.star_surface(6, 20.0, seed=1235)
        mesh = b.Mesh(V, T, b.charges_in_star(2000, shape, seed=1236))
        desc = dict(workload="star-shaped molecule R=20 A (l<=6 harmonics, amp 0.15), icosphere k=6 "
                             "(40962 patches), 2000 charges, eps 2/80, kappa 0.1, qual 4 / quad 0, "
                             "FMM order 9, reference tree nbsize 1500", patches=40962)
        return desc, [(mesh, None, (1, 0, 0, 0))], 0.1, 1500
    if name == "star-small":
        V, T, shape = b.star_surface(5, 20.0, seed=1235)
        mesh = b.Mesh(V, T, b.charges_in_star(500, shape, seed=1236))
        desc = dict(workload="star-shaped molecule R=20 A, icosphere k=5 (10242 patches), 500 charges, eps 2/80, "
                             "kappa 0.1, qual 4 / quad 0, FMM order 9, reference tree nbsize 1500 "
                             "(profiling case)", patches=10242)
        return desc, [(mesh, None, (1, 0, 0, 0))], 0.1, 1500
    if name == "star-large":
        V, T, shape = b.star_surface(7, 40.0, seed=1237)
        mesh = b.Mesh(V, T, b.charges_in_star(20000, shape, seed=1238))
        desc = dict(workload="star-shaped molecule R=40 A, icosphere k=7 (163842 patches), 20000 charges, "
                             "eps 2/80, kappa 0.125, qual 4 / quad 0, FMM order 9, reference tree nbsize 1500 "
                             "(config P's size)", patches=163842)
        return desc, [(mesh, None, (1, 0, 0, 0))], 0.125, 1500
    raise ValueError(f"unknown workload {name}")


def build_beep(meshes, kappa, nbsize, precision, device, context=None, tree=None, **opts):
    import beep3_b200 as b
    kw = dict(tree) if tree else dict(nbsize=nbsize)
    bp = b.BEEP(eps_solvent=80.0, kappa=kappa, precision=precision, device=device, context=context, **kw, **opts)
    for mesh, off, q in meshes:
        bp.insert_mesh_instance(mesh, offset=off, rotation=q, eps_protein=2.0)
    bp.build()
    return bp


def tuned_tree(meshes, kappa, nbsize, local, x, y, steps, flush):
    """The tree and near-field storage (FP32 or compact coefficients) the
    autotuner picks for a problem solved many times (100 solves per build)
    on the same molecule, and the mixed matvec/s on it: the performance
    configuration, beside the headline's parity tree and FP32 cache."""
    import beep3_b200 as b
    from beep3_b200.autotune import autotune, problem_trial
    ctx = b.EngineContext(local)
    try:
        def make(**kw):
            bp = b.BEEP(eps_solvent=80.0, kappa=kappa, precision="mixed", device=local, context=ctx, **kw)
            for mesh, off, q in meshes:
                bp.insert_mesh_instance(mesh, offset=off, rotation=q, eps_protein=2.0)
            return bp
        t0 = time.perf_counter()
        res = autotune(problem_trial(make, solves_per_problem=100.0, repeats=2), compact=(False, True))
        tune_s = time.perf_counter() - t0
        bp = build_beep(meshes, kappa, nbsize, "mixed", local, context=ctx, tree=res.settings())
        try:
            time_device_matvecs(bp, x, y, 3, flush)
            ms = time_device_matvecs(bp, x, y, steps, flush)
            inf = bp.info()
            return {"settings": res.settings(), "matvec_per_s": steps / (sum(ms) / 1e3),
                    "ms_per_step": sum(ms) / steps,
                    "energy_rel_vs_parity_tree": abs(res.best.energies[0] - res.reference_energies[0])
                    / abs(res.reference_energies[0]),
                    "nearfield_pairs": int(inf.n_nearfield_pairs), "tree_levels": int(inf.n_levels),
                    "tuning_seconds": tune_s,
                    "trials": [{"tree": t.tree, "size": t.size, "compact": t.compact, "cost_ms": t.cost_ms,
                                "status": t.status}
                               for t in res.trials]}
        finally:
            bp.close()
    finally:
        ctx.close()


def compact_nearfield(meshes, kappa, nbsize, local, x, y, steps, flush, e_fp64, hbm):
    """The mixed engine with the compact near field (BP_FLAG_COMPACT_NEARFIELD:
    coefficients rounded to 24 bits, 12 bytes a pair) on the headline's
    tree: matvec/s, the apply kernel's time and bandwidth, and the energy
    against the FP64 engine's."""
    bp = build_beep(meshes, kappa, nbsize, "mixed", local, compact_nearfield=True)
    try:
        inf = bp.info()
        n2 = 2 * bp.num_patches
        time_device_matvecs(bp, x, y, 3, flush)
        ms = time_device_matvecs(bp, x, y, steps, flush)
        near_ms = stage_profile(bp, x, y)[0][0]
        alg = inf.n_nearfield_pairs * 12 + inf.n_nearfield_cols * 4 + n2 * 8 * 2 + bp.num_patches * 32
        bp.solve(1e-6, 100)
        e, _ = bp.calculate_energies()
        return {"matvec_per_s": steps / (sum(ms) / 1e3), "ms_per_step": sum(ms) / steps,
                "apply_ms": near_ms, "apply_algorithmic_bytes": int(alg),
                "apply_gbs": alg / (near_ms * 1e-3) / 1e9, "apply_frac": alg / (near_ms * 1e-3) / 1e9 / hbm,
                "device_bytes": int(inf.device_bytes),
                "energy_rel_vs_fp64": abs(e - e_fp64) / abs(e_fp64),
                "note": "near-field coefficients rounded to 24 bits (at most 2^-16 relative each), "
                        "12 bytes a pair; an option of this engine, not the reference's FP32 cache"}
    finally:
        bp.close()


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- helpers
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def allreduce_max(dist, v: float, device) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_device_matvecs(bp, x, y, steps: int, flush) -> list[float]:
    """Per-step device time (ms) of bp_matvec_device with CUDA events on the
    engine's stream; L2 flushed between steps (outside the events) when the
    working set fits in L2."""
    import torch
    from beep3_b200 import _native as N
    L = N.lib()
    p = bp.build()
    stream = torch.cuda.current_stream()
    assert stream.cuda_stream != 0, "time on a non-default stream"
    N.check(L.bp_ctx_set_stream(bp.context(), C.c_void_p(stream.cuda_stream)))
    out = []
    for _ in range(steps):
        if flush is not None:
            flush.add_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        N.check(L.bp_matvec_device(p, x.data_ptr(), y.data_ptr()))
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def time_e2e(bp, xh, yh, steps: int) -> list[float]:
    """Per-step time (ms) of the host-buffer ABI call bp_matvec, bracketed by
    CUDA events on the engine's stream (the call copies x in and y out)."""
    import torch
    from beep3_b200 import _native as N
    L = N.lib()
    p = bp.build()
    stream = torch.cuda.current_stream()
    N.check(L.bp_ctx_set_stream(bp.context(), C.c_void_p(stream.cuda_stream)))
    out = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        N.check(L.bp_matvec(p, xh.data_ptr(), yh.data_ptr()))
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def stage_profile(bp, x, y, reps: int = 5):
    from beep3_b200 import _native as N
    ms = np.zeros(8)
    launches = np.zeros(8, np.int32)
    ns = C.c_int32()
    N.check(N.lib().bp_matvec_profile(bp.build(), x.data_ptr(), y.data_ptr(), reps, N.ptr(ms), N.ptr(launches),
                                      C.byref(ns)))
    return ms, launches


def child_line(local: int, args: list, keys: tuple) -> dict:
    """One bench mode run in a child process on the same GPU: the chosen
    keys of its JSON line, or the reason it has none."""
    cmd = [sys.executable, str(Path(__file__).resolve())] + args
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env)
        d = json.loads(out.stdout.strip().splitlines()[-1])
        return {k: d[k] for k in keys if k in d}
    except Exception as e:  # the headline line stands without it
        return {"unavailable": f"{type(e).__name__}: {e}"[:300]}


def scan_child(local: int) -> dict:
    """Config B's batched rigid-body scan (64 poses of the two star
    molecules, 4 workers x 4 poses per batch problem, the meshes keeping
    their own close pairs' coefficients)."""
    return child_line(local, ["--workload", "scan", "--workers", "4", "--batch", "4", "--cache-pairs"],
                      ("value", "unit", "seconds", "mean_iterations", "config"))


def serve_child(local: int) -> dict:
    """Config R's served request stream (Poisson arrivals, 2562-163842
    patches, admission by HBM budget)."""
    return child_line(local, ["--workload", "serve"],
                      ("value", "unit", "latency_ms", "seconds", "requests", "config"))


def matvec_roofline(inf, n, mv_ms, near_ms, stage_ms, hbm, peaks):
    """The whole matvec against HBM with its algorithmic bytes,
    B_mv = P_nf (16 B coefficients + 4 B column id) + 4N x 8 B (x, y) + B_fmm,
    B_fmm = nodes x 12 channels x (2 x E x 8 B (M, L read + write) + 6 x np x
    2 x 8 B (plane waves written and read)), FP32 complex; and the far field
    alone: its time in the graph (the matvec minus the near field, which
    runs after it), its bytes, and the flops of its operator GEMMs (M->X and
    wave->local, 12 np x 2E real MACs per column, three TF32 passes each)
    against the stage times that hold them."""
    E, NP = int(inf.fmm_coefficients), int(inf.fmm_plane_waves)
    b_fmm = int(inf.n_nodes) * 12 * (2 * E * 8 + 6 * NP * 2 * 8) if inf.fmm_active else 0
    b_mv = int(inf.n_nearfield_pairs) * 20 + 4 * n * 8 + b_fmm
    far_ms = max(mv_ms - near_ms, 1e-9)
    gemm_flops = 2.0 * (int(inf.fmm_m2x_cols) + int(inf.fmm_x2l_cols)) * (12 * NP) * (2 * E)
    xl_flops = 8.0 * int(inf.fmm_translations) * 12 * NP
    shift_flops = 2.0 * int(inf.fmm_shift_cols) * (2 * E) ** 2
    gemm_stage_ms = float(stage_ms[3] + stage_ms[4])  # M->X and X->L (translations + wave->local) stages
    tf32 = float(peaks.get("bf16_tflops", 1590.0)) / 2.0
    achieved_tf = 3 * gemm_flops / (gemm_stage_ms * 1e-3) / 1e12 if gemm_stage_ms > 0 else 0.0
    return {
        "bound": "hbm", "unit": "GB/s", "algorithmic_bytes": b_mv, "achieved": b_mv / (mv_ms * 1e-3) / 1e9,
        "peak": hbm, "frac": b_mv / (mv_ms * 1e-3) / 1e9 / hbm,
        "far_field": {
            "ms_in_graph": far_ms, "algorithmic_bytes": b_fmm,
            "achieved_gbs": b_fmm / (far_ms * 1e-3) / 1e9, "frac_hbm": b_fmm / (far_ms * 1e-3) / 1e9 / hbm,
            "flops": {"operator_gemms": gemm_flops, "translations": xl_flops, "shifts": shift_flops},
            "operator_gemm_tflops_3xtf32": achieved_tf, "tf32_peak_tflops": tf32,
            "operator_gemm_frac": achieved_tf / tf32,
            "note": "far-field time = matvec - near field (the near field runs after the far field); GEMM rate "
                    "over the serialised M->X and X->L stage times, which also hold the translations; TF32 "
                    "peak = half the measured bf16 burst",
        },
    }


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def oracle_timings(arr, tree, charges, kappa: float, edge: float, nterms: int, eps_solvent: float,
                   matvec_budget_s: float, steps: int | None = None, warmup: int = 0) -> dict:
    """The reference's CPU path restated by the oracle (-march=native build,
    OpenMP over the loops the reference parallelises), timed on this host:
    the near-field precalc (once), matvecs (``steps`` of them after
    ``warmup``, or as many as fit in ``matvec_budget_s``), and one full solve
    with its right-hand side timed apart.  Returns the timings and the
    oracle problem (the caller closes it)."""
    import oracle as O
    O.use_native()
    t0 = time.perf_counter()
    pr = O.Problem(arr, tree, kappa, fp32=True, cube_edge=edge, nterms=nterms)
    precalc_s = time.perf_counter() - t0
    x = np.random.default_rng(5).standard_normal(2 * pr.n)
    for _ in range(warmup):
        pr.matvec(x)
    times = []
    while (len(times) < steps) if steps else (sum(times) < matvec_budget_s and len(times) < 1000):
        t = time.perf_counter()
        pr.matvec(x)
        times.append(time.perf_counter() - t)
    t = time.perf_counter()
    rhs = O.rhs(pr.patches, charges, eps_solvent)
    rhs_s = time.perf_counter() - t
    t = time.perf_counter()
    xs, its, rr = pr.solve(rhs, 1e-6, 100)
    gmres_s = time.perf_counter() - t
    return dict(problem=pr, x=x, rhs=rhs, solution=xs, iterations=its, precalc_s=precalc_s, matvec_s=times,
                rhs_s=rhs_s, gmres_s=gmres_s)


def cpu_record(t: dict, kind: str = "port") -> dict:
    mv = len(t["matvec_s"]) / sum(t["matvec_s"])
    return {"value": mv, "unit": "matvec/s", "cores": cpu_threads(), "kind": kind,
            "sample": f"{len(t['matvec_s'])} matvecs of the full workload ({sum(t['matvec_s']):.1f} s) by the "
                      f"oracle's restatement of the reference CPU path (cached FP32 near field + FP64 plane-wave "
                      f"FMM, OpenMP, -O3 -march=native); near-field precalc, right-hand side and GMRES timed once",
            "matvec_ms": 1e3 / mv, "precalc_s": t["precalc_s"], "rhs_s": t["rhs_s"], "gmres_s": t["gmres_s"],
            "gmres_iterations": t["iterations"], "solves_per_s": 1.0 / (t["rhs_s"] + t["gmres_s"]),
            "solves_per_s_gmres_only": 1.0 / t["gmres_s"],
            "note": "the right-hand side is a direct FP64 sum (the reference's is a 6-figure FMM); "
                    "solves_per_s counts right-hand side + GMRES on a built problem, as the engine's does"}


def cpu_baseline_and_parity(bp, bp64, budget_s: float = 12.0) -> tuple[dict, dict]:
    """CPU baseline on the benchmark's problem (same tree and inputs), and the
    engines' parity against the oracle on it: the mixed engine against the
    reference-faithful oracle (matvec, solved f/h, energy), and both engines'
    matvec rows against the FP64 direct-sum oracle on 1024 targets."""
    import oracle as O
    arr = bp.gathered()
    tree = bp.host_tree()
    _, edge = bp.calculate_bounding_cube()
    inst = bp.instances[0]
    t = oracle_timings(arr, tree, inst.charges, bp.kappa, edge, bp.nterms, bp.eps_solvent, budget_s)
    pr, x = t["problem"], t["x"]
    n = pr.n
    try:
        yo = pr.matvec(x)
        ym, y64 = bp.matvec(x), bp64.matvec(x)
        ecf, ech = O.energy_coefficients(arr["gal_off"], arr["gal"], arr["area"], inst.charges,
                                         inst.mesh.patches.total_area)
        xo = t["solution"]
        eo = O.energy(xo[:n], xo[n:], ecf, ech, inst.dielectric_ratio)
        em, _ = bp.calculate_energies()
        targets = np.random.default_rng(6).choice(n, 1024, replace=False)
        ex = O.exact_rows(arr, tree, bp.kappa, x, targets)
        mf, mh = O.row_errors(ym, ex, targets, n)
        df, dh = O.row_errors(y64, ex, targets, n)
        of, oh = O.row_errors(yo, ex, targets, n)
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        parity = {
            "error_vs_oracle": {
                "what": "mixed engine against the oracle (the reference's CPU path restated: FP32 near-field "
                        "coefficients, FP64 FMM) on the same tree and inputs",
                "matvec_rel_l2": rel(ym, yo), "solution_f_rel_l2": rel(bp.x[:n], xo[:n]),
                "solution_h_rel_l2": rel(bp.x[n:], xo[n:]), "energy_rel": abs(em - eo) / abs(eo),
                "gmres_iterations_oracle": t["iterations"]},
            "error_vs_direct": {
                "what": "matvec rows on 1024 random target patches against the FP64 direct-sum oracle (every "
                        "near pair in FP64, far field summed exactly): the order-9 FMM's truncation",
                "mixed_f": mf, "mixed_h": mh, "fp64_f": df, "fp64_h": dh, "oracle_fmm_f": of, "oracle_fmm_h": oh}}
    finally:
        pr.close()
    return cpu_record(t), parity


# --------------------------------------------------------------------------- arms
def prepare_inputs(name: str, path: str) -> None:
    """Writes the workload's gathered patch arrays, charges and bounding cube
    to ``path`` (npz).  Run in a child process of the reference arm, so the
    reference arm's own process never loads the engine library (the surface
    point generation is the engine's host geometry code)."""
    desc, meshes, kappa, nbsize = workload(name)
    import beep3_b200 as b
    bp = b.BEEP(eps_solvent=80.0, kappa=kappa, nbsize=nbsize, precision="mixed")
    for mesh, off, q in meshes:
        bp.insert_mesh_instance(mesh, offset=off, rotation=q, eps_protein=2.0)
    arr = bp.gathered()
    centre, edge = bp.calculate_bounding_cube()
    charges = np.concatenate([i.charges for i in bp.instances])
    np.savez(path, **{k: v for k, v in arr.items() if k != "first"}, charges=charges, centre=centre,
             edge=edge, kappa=kappa, nbsize=nbsize, nterms=bp.nterms, eps_solvent=bp.eps_solvent,
             desc=json.dumps(desc))


def run_reference(args):
    world, rank, local, dist = dist_setup(args)
    if rank != 0:
        return
    if args.workload in ("scan", "serve"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the matvec workloads only"}),
              flush=True)
        return
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "inputs.npz")
        subprocess.run([sys.executable, str(Path(__file__).resolve()), "--prepare-inputs", path, "--workload",
                        args.workload], check=True)
        z = np.load(path)
        arr = {k: z[k] for k in ("centroid", "normal", "area", "eps", "gc", "qual_off", "qual", "quad_off", "quad",
                                 "gal_off", "gal")}
        charges, centre, edge = z["charges"], z["centre"], float(z["edge"])
        kappa, nbsize, nterms = float(z["kappa"]), int(z["nbsize"]), int(z["nterms"])
        eps_solvent, desc = float(z["eps_solvent"]), json.loads(str(z["desc"]))
    from oracle import tree as OT
    tree = OT.build(arr["centroid"], centre, edge, nbsize)
    t = oracle_timings(arr, tree, charges, kappa, edge, nterms, eps_solvent, 0.0, steps=args.steps,
                       warmup=args.warmup)
    t["problem"].close()
    rec = cpu_record(t)
    val = rec["value"]
    tot = sum(t["matvec_s"])
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "matvec/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32 near field/fp64 FMM",
            "data": "synthetic", "config": desc, "cpu_baseline": rec,
            "e2e": {"value": val, "unit": "matvec/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "engine_library_loaded": any("libbeep3_b200" in ln for ln in Path("/proc/self/maps").read_text()
                                         .splitlines())}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    world, rank, local, dist = dist_setup(args)
    torch.cuda.set_device(local)
    # a dedicated (non-default) stream: the engine and the CUDA events of the
    # timing run on it (the legacy default stream has handle 0, which the
    # engine's bp_ctx_set_stream reads as "its own stream")
    with torch.cuda.stream(torch.cuda.Stream()):
        _run_ours(args, world, rank, local, dist)


def _only_matvec(args, local):
    """Profiling mode: the mixed engine only, W warm-up + K timed matvecs."""
    import torch
    desc, meshes, kappa, nbsize = workload(args.workload)
    bp = build_beep(meshes, kappa, nbsize, "mixed", local, compact_nearfield=args.compact)
    dev = torch.device("cuda", local)
    x = torch.randn(2 * bp.num_patches, dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    time_device_matvecs(bp, x, y, args.warmup, None)
    ms = time_device_matvecs(bp, x, y, args.steps, None)
    print(json.dumps({"mode": "only-matvec", "config": desc, "compact_nearfield": args.compact,
                      "ms_per_step": sum(ms) / len(ms)}), flush=True)
    bp.close()


def _scan_mode(args, local):
    """Batched rigid-body scan: two star molecules (40962 and 10242 patches,
    different seeds) over random poses (uniform quaternion, centre separation
    uniform in 45-80 A), each pose's complex solved and its interaction
    energy taken; poses run concurrently on their own engine contexts."""
    import beep3_b200 as b
    from beep3_b200.scan import random_poses, rigid_body_scan
    va, ta, sa = b.star_surface(6, 20.0, seed=1235)
    ma = b.Mesh(va, ta, b.charges_in_star(2000, sa, seed=1236))
    vb, tb, sb = b.star_surface(5, 20.0, seed=2235)
    mb = b.Mesh(vb, tb, b.charges_in_star(500, sb, seed=2236))
    poses = random_poses(args.poses, seed=1237)
    # one engine context per worker, kept across scans: the meshes and the
    # device blocks of a pose stay on the device for the next
    ctxs = [b.EngineContext(local) for _ in range(args.workers)]
    tree = 1500  # the reference's nbsize
    if args.compact:
        tree = dict(nbsize=1500, compact_nearfield=True)
    tuned = None
    try:
        snap = not args.exact_cubes
        if args.autotune:
            # the tree chosen by short scans of 16 other poses in the same
            # worker / batch configuration, outside the timed scans (energies
            # within 1e-4 of the reference tree's)
            from beep3_b200.autotune import autotune
            from beep3_b200.scan import scan_trial
            tune_poses = random_poses(16, seed=98)
            rigid_body_scan(ma, mb, tune_poses, kappa=0.1, workers=args.workers, device=local, contexts=ctxs,
                            snap_cube_edges=snap, batch=args.batch)
            t0 = time.perf_counter()
            res_t = autotune(scan_trial(ma, mb, tune_poses, kappa=0.1, workers=args.workers, batch=args.batch,
                                        device=local, contexts=ctxs, snap_cube_edges=snap))
            tuned = {"settings": res_t.settings(), "seconds": time.perf_counter() - t0,
                     "trials": [{"tree": t.tree, "size": t.size, "ms_per_pose": t.cost_ms, "status": t.status}
                                for t in res_t.trials]}
            tree = res_t.settings()
        # warm-up: a scan of as many other poses, so that every context has
        # seen problems of the sizes the timed scan builds
        rigid_body_scan(ma, mb, random_poses(args.poses, seed=99), kappa=0.1, workers=args.workers, device=local,
                        contexts=ctxs, snap_cube_edges=snap, batch=args.batch, nbsize=tree,
                        cache_pairs=args.cache_pairs, warm_start=args.warm_start)
        # a scan of 64 poses lasts about a second, and host threads make it
        # vary from run to run: the median of three timed scans
        runs = [rigid_body_scan(ma, mb, poses, kappa=0.1, workers=args.workers, device=local, contexts=ctxs,
                                snap_cube_edges=snap, batch=args.batch, nbsize=tree, cache_pairs=args.cache_pairs,
                                warm_start=args.warm_start)
                for _ in range(3)]
        runs.sort(key=lambda r: r.poses_per_s)
        res = runs[1]
    finally:
        for c in ctxs:
            c.close()
    e = np.asarray(res.energies)
    print(json.dumps({
        "metric": "rigid-body scan poses/s (mixed engine, full solve + interaction energy per pose)",
        "value": res.poses_per_s, "unit": "poses/s", "n_gpus": 1, "higher_is_better": True,
        "data": "synthetic", "dtype": "fp32 near field/FMM + fp64 singular/GMRES",
        "config": {"workload": "batched rigid-body scan: star k=6 (40962 patches, 2000 charges) + star k=5 "
                               "(10242 patches, 500 charges), kappa 0.1, separation 45-80 A",
                   "poses": len(poses), "workers": args.workers,
                   "poses_per_batch": args.batch,
                   "engine_contexts": "one per worker, kept across scans",
                   "mesh_pair_cache": bool(args.cache_pairs),
                   "compact_nearfield": bool(args.compact),
                   "warm_start": bool(args.warm_start),
                   "cube_edges": "exact per pose" if args.exact_cubes else
                                 "rounded up to 2^(k/8): poses share far-field plans"},
        "seconds": res.seconds, "mean_iterations": float(np.mean(res.iterations)),
        "timed_scans_poses_per_s": [r.poses_per_s for r in runs], "value_is": "median of the timed scans",
        "tree": tree, "autotune": tuned,
        "interaction_energy_kj_per_mol": {"min": float(e.min()), "max": float(e.max()), "mean": float(e.mean())},
    }), flush=True)


def _serve_mode(args, local):
    """Served request stream: Poisson arrivals of single-molecule solves,
    patch counts log-uniform in 2562-163842 (snapped to icosphere levels
    4-7, radius scaled with the patch count), charges 0.05 x patches, kappa
    from {0, 0.05, 0.1, 0.15}; admission by HBM budget with worker slots."""
    import beep3_b200 as b
    from beep3_b200.server import BemServer, SolveRequest
    rng = np.random.default_rng(4321)
    levels = {2562: 4, 10242: 5, 40962: 6, 163842: 7}
    sizes = np.array(sorted(levels))
    meshes = {}
    plan = []
    for r in range(args.requests):
        n = float(np.exp(rng.uniform(np.log(2562), np.log(163842))))
        n_snap = int(sizes[np.argmin(np.abs(np.log(sizes) - np.log(n)))])
        kappa = float(rng.choice([0.0, 0.05, 0.1, 0.15]))
        plan.append((n_snap, kappa, float(rng.exponential(1.0 / args.rate))))
        if n_snap not in meshes:
            k = levels[n_snap]
            v, t, shape = b.star_surface(k, 20.0 * (n_snap / 40962) ** 0.5, seed=5000 + k)
            meshes[n_snap] = b.Mesh(v, t, b.charges_in_star(int(0.05 * n_snap), shape, seed=6000 + k))
    tree_for = None
    if args.serve_device_tree_from:  # the device-built tree (cap 128) for requests of at least this size
        cut = args.serve_device_tree_from
        tree_for = lambda n: dict(tree="device", leaf_size=128) if n >= cut else dict(nbsize=1500)
    srv = BemServer(device=local, workers=args.workers, tree_for=tree_for)
    try:
        # warm-up: the same stream once, untimed, so that the slots' engine
        # contexts hold the meshes and far-field plans a running server would
        wfuts = []
        for n_snap, kappa, gap in plan:
            time.sleep(gap)
            wfuts.append(srv.submit(SolveRequest(meshes[n_snap], kappa, tag=n_snap)))
        for f in wfuts:
            f.result()
        futs = []
        t0 = time.perf_counter()
        for n_snap, kappa, gap in plan:
            time.sleep(gap)
            futs.append(srv.submit(SolveRequest(meshes[n_snap], kappa, tag=n_snap)))
        results = [f.result() for f in futs]
        wall = max(r.end for r in results) - t0
    finally:
        srv.close()
    lat = np.array([r.latency_ms for r in results])
    print(json.dumps({
        "metric": "served solves/s and p50/p99 latency (mixed engine, continuous batching)",
        "value": len(results) / wall, "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
        "data": "synthetic", "dtype": "fp32 near field/FMM + fp64 singular/GMRES",
        "config": {"workload": "served stream: Poisson arrivals, star surfaces of 2562-163842 patches "
                               "(log-uniform), charges 0.05 x patches, kappa in {0, 0.05, 0.1, 0.15}",
                   "requests": len(results), "rate_per_s": args.rate, "worker_slots": args.workers,
                   "tree": ("device tree, cap 128, from %d patches" % args.serve_device_tree_from
                            if args.serve_device_tree_from else "reference tree, nbsize 1500")},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max())},
        "all_converged": all(r.converged for r in results),
        "peak_device_bytes_admitted": srv.peak_in_use,
        "patches": {str(k): int(sum(1 for r in results if r.n_patches == k)) for k in sorted(meshes)},
    }), flush=True)


def _run_ours(args, world, rank, local, dist):
    import torch
    if args.only_matvec:
        _only_matvec(args, local)
        return
    if args.workload in ("scan", "serve"):
        if rank == 0:
            (_scan_mode if args.workload == "scan" else _serve_mode)(args, local)
        return
    from beep3_b200 import _native as N
    dev = torch.device("cuda", local)
    desc, meshes, kappa, nbsize = workload(args.workload)
    bp = build_beep(meshes, kappa, nbsize, "mixed", local)
    bp64 = build_beep(meshes, kappa, nbsize, "fp64", local)
    n2 = 2 * bp.num_patches
    inf = bp.info()
    gen = torch.Generator(device="cpu").manual_seed(7)
    x = torch.randn(n2, dtype=torch.float64, generator=gen).to(dev)
    y = torch.empty_like(x)
    working = inf.n_nearfield_pairs * 16 + n2 * 16
    flush = torch.zeros(2 * L2_BYTES // 4, dtype=torch.float32, device=dev) if working < 2 * L2_BYTES else None
    # warm-up
    time_device_matvecs(bp, x, y, max(args.warmup, 3), flush)
    time_device_matvecs(bp64, x, y, max(args.warmup, 3), flush)
    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    steps_ms = time_device_matvecs(bp, x, y, args.steps, flush)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    t_local = sum(steps_ms)
    t_max = allreduce_max(dist, t_local, dev)
    value = world * args.steps / (t_max / 1e3)
    # FP64 engine, same steps
    steps64 = time_device_matvecs(bp64, x, y, args.steps, flush)
    t64 = allreduce_max(dist, sum(steps64), dev)
    value64 = world * args.steps / (t64 / 1e3)
    # end to end through the host-buffer ABI
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    time_e2e(bp, xh, yh, 3)
    e2e_ms = time_e2e(bp, xh, yh, args.steps)
    te = allreduce_max(dist, sum(e2e_ms), dev)
    e2e_value = world * args.steps / (te / 1e3)
    # stage profile -> roofline of the dominant kernel (near-field apply)
    ms, launches = stage_profile(bp, x, y)
    near_ms = ms[0]
    alg_bytes = inf.n_nearfield_pairs * 16 + inf.n_nearfield_cols * 4 + n2 * 8 * 2 + bp.num_patches * 32
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (near_ms * 1e-3) / 1e9
    # solves (RHS + GMRES) and energies, both precisions
    solve_ms, solve64_ms, rhs_ms, gmres_ms = [], [], [], []
    for _ in range(3):
        bp.solve(1e-6, 100)
        bp64.solve(1e-6, 100)
    for _ in range(max(3, args.steps // 4)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        info = bp.solve(1e-6, 100)
        solve_ms.append((time.perf_counter() - t) * 1e3)
        rhs_ms.append(info.time_rhs_ms)
        gmres_ms.append(info.time_gmres_ms)
        t = time.perf_counter()
        info64 = bp64.solve(1e-6, 100)
        solve64_ms.append((time.perf_counter() - t) * 1e3)
    # GMRES alone on device arrays (bp_solve_device, x0 = 0): its time beyond
    # the matvecs it runs (one per iteration) is the solver's own overhead
    rhs_d = torch.tensor(bp.set_rhs(), device=dev)
    gm_ms = []
    for r in range(3 + max(3, args.steps // 4)):
        x_d = torch.zeros_like(rhs_d)
        its_c, rr_c = C.c_int32(), C.c_double()
        torch.cuda.synchronize()
        t = time.perf_counter()
        N.check(N.lib().bp_solve_device(bp.build(), rhs_d.data_ptr(), x_d.data_ptr(), 1e-6, 100, 0,
                                        C.byref(its_c), C.byref(rr_c)))
        torch.cuda.synchronize()
        if r >= 3:
            gm_ms.append((time.perf_counter() - t) * 1e3)
    gmres_dev_ms = float(np.median(gm_ms))
    e_mixed, _ = bp.calculate_energies()
    e_fp64, _ = bp64.calculate_energies()
    line = {
        "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32 near field/FMM + fp64 singular/GMRES", "data": "synthetic",
        "config": dict(desc, precision="mixed", parallelism=f"replicas x{world}",
                       l2="flushed between steps" if flush is not None else "inputs larger than L2",
                       nearfield_pairs=int(inf.n_nearfield_pairs), tree_levels=int(inf.n_levels),
                       fmm=bool(inf.fmm_active)),
        "e2e": {"value": e2e_value, "unit": "matvec/s", "h2d_bytes_per_step": n2 * 8, "d2h_bytes_per_step": n2 * 8},
        "gpu_launches": int(launches.sum()) * args.steps,
        "roofline": {"bound": "hbm", "kernel": "nearfield apply_kernel<float>", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "traffic": APPLY_TRAFFIC.get(args.workload),
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback",
                     "algorithmic_bytes_per_launch": int(alg_bytes), "launch_ms": near_ms},
        "roofline_matvec": matvec_roofline(inf, bp.num_patches, t_max / args.steps, near_ms, ms, hbm, peaks),
        "stage_ms": {k: round(float(v), 5) for k, v in zip(
            ["near+add", "p2m", "m2m", "m2x", "x2l", "l2p_prep", "l2l", "l2p_eval"], ms)},
        "fp64_matvec_per_s": value64,
        "fp64_stage_ms": {k: round(float(v), 5) for k, v in zip(
            ["near+add", "p2m", "m2m", "m2x", "x2l", "l2p_prep", "l2l", "l2p_eval"], stage_profile(bp64, x, y)[0])},
        "mixed_over_fp64": value / value64,
        "solves_per_s": world * 1e3 / statistics.median(solve_ms),
        "fp64_solves_per_s": world * 1e3 / statistics.median(solve64_ms),
        "solve_latency_ms": {"p50": float(np.percentile(solve_ms, 50)), "p99": float(np.percentile(solve_ms, 99))},
        "solve_parts_ms": {"rhs": float(np.median(rhs_ms)), "gmres": float(np.median(gmres_ms))},
        "gmres_iterations": {"mixed": info.num_iterations, "fp64": info64.num_iterations},
        "gmres_device": {"ms": gmres_dev_ms, "iterations": its_c.value,
                         "overhead_ms": gmres_dev_ms - its_c.value * t_max / args.steps,
                         "note": "bp_solve_device from x = 0 (no matvec for the first residual): time minus "
                                 "iterations x the timed matvec"},
        "gmres_loop_on_device": bool(bp.info().gmres_graph),
        "energy_kj_per_mol": {"mixed": e_mixed, "fp64": e_fp64,
                              "rel_err_mixed_vs_fp64": abs(e_mixed - e_fp64) / abs(e_fp64)},
        "clocks": clocks,
    }
    if rank == 0 and world == 1:
        try:  # an extra key: the headline line stands without it
            line["compact_nearfield"] = compact_nearfield(meshes, kappa, nbsize, local, x, y, args.steps, flush,
                                                          e_fp64, hbm)
        except Exception as e:
            line["compact_nearfield"] = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:  # the CPU baseline: rank 0 at N = 1 only
        line["cpu_baseline"], parity = cpu_baseline_and_parity(bp, bp64)
        line.update(parity)
    if rank == 0 and world == 1 and not args.no_scan and args.workload == "star":
        try:  # an extra key: the headline line stands without it
            line["tuned_tree"] = tuned_tree(meshes, kappa, nbsize, local, x, y, args.steps, flush)
        except Exception as e:
            line["tuned_tree"] = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
        line["scan_config_b"] = scan_child(local)
        line["serve_config_r"] = serve_child(local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    bp.close()
    bp64.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="star",
                    choices=["kirkwood", "star", "star-small", "star-large", "scan", "serve"],
                    help="scan / serve: the batched rigid-body scan and the served request stream")
    ap.add_argument("--poses", type=int, default=64, help="scan: number of poses")
    ap.add_argument("--autotune", action="store_true",
                    help="scan: choose the tree by short measured scans before the timed scans")
    ap.add_argument("--batch", type=int, default=1,
                    help="scan: poses solved together as the scenarios of one batch problem")
    ap.add_argument("--requests", type=int, default=24, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=8.0, help="serve: Poisson arrival rate, requests/s")
    ap.add_argument("--serve-device-tree-from", type=int, default=100000,
                    help="serve: requests of at least this many patches use the device-built tree (cap 128), "
                         "whose set-up is half the reference tree's at 163842 patches; 0: the reference tree "
                         "for all")
    ap.add_argument("--workers", type=int, default=4, help="scan / serve: concurrent solves")
    ap.add_argument("--only-matvec", action="store_true", help="profiling mode: matvecs of the mixed engine only")
    ap.add_argument("--warm-start", action="store_true",
                    help="scan: every pose's GMRES starts from the isolated molecules' solutions")
    ap.add_argument("--cache-pairs", action="store_true",
                    help="scan: the meshes keep their own close pairs' near-field coefficients")
    ap.add_argument("--compact", action="store_true",
                    help="profiling and scan modes: the compact (24-bit) near-field coefficients")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-scan", action="store_true",
                    help="leave out the config-B scan and config-R serving keys of the default line")
    ap.add_argument("--exact-cubes", action="store_true",
                    help="scan: each pose's exact bounding cube (no far-field plan sharing)")
    ap.add_argument("--prepare-inputs", metavar="NPZ", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.prepare_inputs:
        prepare_inputs(args.workload, args.prepare_inputs)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
