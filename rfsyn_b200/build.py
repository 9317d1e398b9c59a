"""Builds librfsyn_fdtd_b200.so in-tree (rfsyn_b200/lib/).

Host C sources are compiled with gcc (C11, no FP contraction, so the host
side evaluates CPML profiles, material coefficients and source samples with
exactly the arithmetic of rfsyn's CPU code); the CUDA engine is compiled
with nvcc for sm_100a only.  Run:  python -m rfsyn_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIBNAME = "librfsyn_fdtd_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIBDIR.mkdir(exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    headers = list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    c_srcs = sorted((CSRC / "host").glob("*.c"))
    cu_srcs = sorted(CSRC.glob("*.cu"))
    objs = []
    for src in c_srcs:
        obj = objdir / (src.stem + ".o")
        if force or _stale(obj, [src] + headers):
            _run(["gcc", "-std=c11", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
                  "-D_GNU_SOURCE", f"-I{ROOT / 'include'}", "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    nvcc = _nvcc()
    for src in cu_srcs:
        obj = objdir / (src.stem + ".cu.o")
        if force or _stale(obj, [src] + headers):
            _run([nvcc, "-std=c++17", *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-diag-suppress", "550",
                  f"-I{ROOT / 'include'}", "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    lib = LIBDIR / LIBNAME
    if force or _stale(lib, objs):
        _run([nvcc, "-shared", *ARCH, "-cudart", "static", "-o", str(lib), *map(str, objs), "-lm"])
    if verbose:
        print(f"built {lib}")
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
