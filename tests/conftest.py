"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device (B200); the rest
run on the CPU (oracle, geometry, tree, ABI loading, host logic)."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    """True when the CUDA driver reports at least one device."""
    import ctypes
    try:
        cuda = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return False
    if cuda.cuInit(0) != 0:
        return False
    n = ctypes.c_int(0)
    return cuda.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0


def pytest_collection_modifyitems(config, items):
    # gpu tests fail loudly on a GPU box; on a CPU-only box they are skipped
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def kirkwood_case():
    """Kirkwood sphere: radius 10, icosphere k=3 (642 patches), 10 charges in
    r < 7 with q ~ U[-1, 1], eps 2/80, kappa 0.1, qual 4 / quad 0."""
    import beep3_b200 as b
    V, T = b.icosphere(3, 10.0)
    ch = b.charges_in_sphere(10, 7.0, seed=1234)
    mesh = b.Mesh(V, T, ch)
    return dict(V=V, T=T, charges=ch, mesh=mesh, kappa=0.1, eps_in=2.0, eps_out=80.0, radius=10.0)


def make_beep(mesh, kappa=0.1, nbsize=1500, precision="fp64", eps_out=80.0, eps_in=2.0, **kw):
    import beep3_b200 as b
    bp = b.BEEP(eps_solvent=eps_out, kappa=kappa, nbsize=nbsize, precision=precision, **kw)
    bp.insert_mesh_instance(mesh, eps_protein=eps_in)
    return bp


def rel_l2(a, b) -> float:
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
