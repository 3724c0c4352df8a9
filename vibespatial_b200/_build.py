"""Build ``libvsjoin.so`` in-tree with nvcc for sm_100a.

``python -m vibespatial_b200._build`` (or ``__graft_entry__.build()``) compiles
every ``csrc/*.cu`` into ``vibespatial_b200/_lib/libvsjoin.so``.  The library
is a plain C-ABI shared object (no torch or Python types in its signatures).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libvsjoin.so"
INCLUDE = PKG.parent / "include"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and not _stale():
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    objdir = PKG.parent / "_build"
    objdir.mkdir(exist_ok=True)
    # gcc from /usr/bin: the toolchain wrapper on PATH may lack OpenMP specs;
    # nvcc's host compiler only needs plain C++17.
    env = dict(os.environ)
    host_cc = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else None
    base = [nvcc(), *NVCC_FLAGS, *(extra or [])]
    if host_cc:
        base += ["-ccbin", host_cc]
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [*base, "-c", str(src), "-o", str(obj), "-I", str(INCLUDE)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)
        objs.append(str(obj))
    link = [*base, "-shared", "-o", str(LIB), *objs, "-lcudart"]
    r = subprocess.run(link, env=env, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
