"""Builds the in-tree shared library ``beep3_b200/libbeep3_b200.so`` for sm_100a.

Run ``python beep3_b200/build.py`` (by path: importing the package loads the
library it builds).  Object files go
to ``beep3_b200/_build/``; a source newer than its object is recompiled.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libbeep3_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                     "--expt-relaxed-constexpr", "-I", str(INCLUDE)]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-I", str(INCLUDE)]
# per-source nvcc flags: the device mesh generator shares the host
# preparation's surface code and must round as the host does (no FMA)
NVCC_FILE_FLAGS = {"mesh_gen.cu": ["--fmad=false"]}


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build beep3_b200")
    return cand


def _cuda_home() -> Path:
    return Path(_nvcc()).resolve().parent.parent


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def build(verbose: bool = False, extra_nvcc: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    newest_header = max((p.stat().st_mtime for p in _headers()), default=0.0)
    objs = []
    for src in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, newest_header):
            continue
        if src.suffix == ".cu":
            cmd = [nvcc, *NVCC_FLAGS, *NVCC_FILE_FLAGS.get(src.name, []), *(extra_nvcc or []), "-c", str(src), "-o",
                   str(obj)]
        else:
            cmd = ["g++", *CXX_FLAGS, "-I", str(_cuda_home() / "include"), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
               "-Xlinker", "-z,defs", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
