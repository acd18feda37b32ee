"""Test-only native shims, built on demand with g++ into tests/native/_build/."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent


def load(name: str, sources: list[Path]) -> C.CDLL:
    """Builds tests/native/<name>.cpp into a shared library when it or one of
    ``sources`` is newer than the library, and loads it."""
    src = HERE / f"{name}.cpp"
    out = HERE / "_build" / f"lib{name}.so"
    deps = [src, *sources]
    if not out.exists() or any(d.stat().st_mtime > out.stat().st_mtime for d in deps):
        out.parent.mkdir(exist_ok=True)
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", str(ROOT / "include"), "-I",
               str(ROOT / "oracle"), str(src), "-o", str(out)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("test shim build failed:\n" + res.stdout + res.stderr)
    return C.CDLL(str(out))
