"""Serving loop host logic (admission by HBM budget, slots, FIFO) with a fake
runner on the CPU."""
import threading
import time

import pytest

from beep3_b200.server import BemServer, SolveRequest, SolveResult, estimate_device_bytes, latency_percentiles


class FakeMesh:
    def __init__(self, n):
        self.n_patches = n


def test_estimate_monotone():
    a = estimate_device_bytes(2562, 1500, "mixed")
    b = estimate_device_bytes(40962, 1500, "mixed")
    c = estimate_device_bytes(40962, 1500, "fp64")
    assert 0 < a < b < c


def test_admission_respects_budget_and_slots():
    live = {"bytes": 0, "count": 0, "peak_bytes": 0, "peak_count": 0}
    lock = threading.Lock()

    def runner(req, need):
        with lock:
            live["bytes"] += need
            live["count"] += 1
            live["peak_bytes"] = max(live["peak_bytes"], live["bytes"])
            live["peak_count"] = max(live["peak_count"], live["count"])
        start = time.perf_counter()
        time.sleep(0.02)
        with lock:
            live["bytes"] -= need
            live["count"] -= 1
        return SolveResult(req.tag, float(req.mesh.n_patches), 1, True, req.mesh.n_patches, need, req.arrival,
                           start, time.perf_counter())

    budget = 1000
    srv = BemServer(hbm_budget_bytes=budget, workers=3, runner=runner,
                    estimator=lambda r: r.mesh.n_patches)
    sizes = [400, 300, 500, 100, 900, 200, 250, 350]
    futs = [srv.submit(SolveRequest(FakeMesh(s), 0.1, tag=i)) for i, s in enumerate(sizes)]
    res = [f.result(timeout=30) for f in futs]
    srv.close()
    assert [r.tag for r in res] == list(range(len(sizes)))
    assert live["peak_bytes"] <= budget
    assert live["peak_count"] <= 3
    assert srv.peak_in_use <= budget
    # several requests overlapped
    assert live["peak_count"] >= 2
    p = latency_percentiles(res)
    assert p["p99"] >= p["p50"] > 0


def test_errors_propagate():
    def runner(req, need):
        raise RuntimeError("boom")

    srv = BemServer(hbm_budget_bytes=100, workers=1, runner=runner, estimator=lambda r: 10)
    f = srv.submit(SolveRequest(FakeMesh(10), 0.1))
    with pytest.raises(RuntimeError):
        f.result(timeout=10)
    # the slot and budget were released: a second request still runs
    f2 = srv.submit(SolveRequest(FakeMesh(10), 0.1))
    with pytest.raises(RuntimeError):
        f2.result(timeout=10)
    srv.close()


def test_measured_footprint_replaces_the_estimate():
    """A size seen before is admitted by the device bytes its earlier request
    really held, not by the estimator's guess (which here undercounts)."""
    needs = []

    def runner(req, need):
        needs.append(need)
        start = time.perf_counter()
        return SolveResult(req.tag, 0.0, 1, True, req.mesh.n_patches, 3 * req.mesh.n_patches, req.arrival, start,
                           time.perf_counter())

    srv = BemServer(hbm_budget_bytes=10_000, workers=1, runner=runner, estimator=lambda r: r.mesh.n_patches)
    srv.submit(SolveRequest(FakeMesh(100), 0.1)).result(timeout=10)
    assert srv.footprint(SolveRequest(FakeMesh(100), 0.1)) == 300
    srv.submit(SolveRequest(FakeMesh(100), 0.1)).result(timeout=10)
    srv.submit(SolveRequest(FakeMesh(50), 0.1)).result(timeout=10)  # unseen size: the estimate
    srv.close()
    assert needs == [100, 300, 50]


def test_tree_per_request_size_keys_the_measured_footprint():
    """tree_for picks a request's tree by its size; footprints learnt from
    measured device bytes are kept per (size, precision, tree, screened)."""
    def runner(req, need):
        start = time.perf_counter()
        return SolveResult(req.tag, 0.0, 1, True, req.mesh.n_patches, 1000 + req.mesh.n_patches, req.arrival,
                           start, time.perf_counter())

    tree_for = lambda n: dict(tree="device", leaf_size=128) if n >= 100000 else dict(nbsize=1500)
    srv = BemServer(runner=runner, estimator=lambda r: 10, tree_for=tree_for, workers=2)
    try:
        small, large = SolveRequest(FakeMesh(2562), 0.1), SolveRequest(FakeMesh(163842), 0.1)
        assert dict(srv._key(large)[2])["tree"] == "device" and dict(srv._key(small)[2])["nbsize"] == 1500
        srv.submit(small).result()
        srv.submit(large).result()
        assert srv.footprint(small) == 1000 + 2562 and srv.footprint(large) == 1000 + 163842
    finally:
        srv.close()
