"""Builds the engine's CUDA/C++ library in-tree.

Every ``.cu`` and ``.cpp`` file under ``encore_b200/csrc`` is compiled for
sm_100a (``-gencode arch=compute_100a,code=sm_100a``) and linked into
``encore_b200/libencore_b200.so``, which the Python package loads with ctypes.
Objects are rebuilt only when a source or header is newer than them.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libencore_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the engine needs the CUDA 12.9 toolchain")
    return cand


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *headers])


def _compile(src: Path, obj: Path, nvcc: str, verbose_ptxas: bool) -> str:
    if src.suffix == ".cu":
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
               "-Xcompiler", "-fPIC,-O3", "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if verbose_ptxas:
            cmd[1:1] = ["-Xptxas", "-v"]
    else:
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off",
               "-I", str(INCLUDE), "-I", "/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    """Compiles the library if anything changed; returns its path."""
    nvcc = _nvcc()
    OBJ.mkdir(exist_ok=True)
    headers = _headers()
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    jobs = []
    for s in srcs:
        o = OBJ / (s.name + ".o")
        if force or verbose_ptxas or _stale(o, s, headers):
            jobs.append((s, o))
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = [ex.submit(_compile, s, o, nvcc, verbose_ptxas) for s, o in jobs]
            for f in futs:
                logs.append(f.result())
    objs = [OBJ / (s.name + ".o") for s in srcs]
    if force or jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    if verbose_ptxas:
        sys.stderr.write("".join(logs))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
    print(LIB)
