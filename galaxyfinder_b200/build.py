"""Builds libgf.so (the CUDA kernels + C ABI) in-tree for sm_100a.

    python -m galaxyfinder_b200.build          # incremental
    python -m galaxyfinder_b200.build --force  # rebuild everything

Each translation unit under csrc/ is compiled by nvcc for
``arch=compute_100a,code=sm_100a`` with ``-lineinfo``; the objects are
linked into ``galaxyfinder_b200/libgf.so`` and archived into
``galaxyfinder_b200/libgf.a`` (for linking into the reference program).  ``gf_tsc.cu``, ``gf_knn.cu`` and
``gf_bound.cu`` and ``gf_cores.cu`` are compiled with ``--fmad=false`` because their results must reproduce the
reference's separately rounded float/double arithmetic bit for bit.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgf.so"
ARCHIVE = PKG / "libgf.a"  # the same objects, for linking libgf into the reference program
TUNED = PKG / "tuned.json"  # launch parameters chosen by tune.py (-D flags)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NOFMAD = {"gf_tsc.cu", "gf_knn.cu", "gf_bound.cu", "gf_cores.cu", "gf_reftree.cu", "gf_plain64.cu", "gf_plan.cu", "gf_shells.cu",
          "gf_rtidal.cu", "gf_starden.cu"}


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def tuned_params() -> dict:
    """The launch parameters recorded by tune.py (empty: the header defaults)."""
    if TUNED.exists():
        return dict(json.loads(TUNED.read_text()).get("params", {}))
    return {}


def _flags(name: str, params: dict | None = None) -> list[str]:
    f = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O2",
         "-I", str(ROOT / "include"), "-I", str(CSRC), "--expt-relaxed-constexpr"]
    if name in NOFMAD:
        f.append("--fmad=false")
    f += [f"-D{k}={int(v)}" for k, v in sorted((tuned_params() if params is None else params).items())]
    return f


def compile_one(src: Path, obj: Path, params: dict | None = None, verbose: bool = False) -> None:
    cmd = [nvcc(), *_flags(src.name, params), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def link(objs, lib: Path, verbose: bool = False) -> None:
    cmd = [nvcc(), "-shared", *ARCH, "-o", str(lib), *map(str, objs), "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    headers = list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    if TUNED.exists():
        headers.append(TUNED)
    newest_header = max((h.stat().st_mtime for h in headers), default=0.0)
    objs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        if not stale:
            continue
        compile_one(src, obj, verbose=verbose)
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        link(objs, LIB, verbose)
    if force or not ARCHIVE.exists() or ARCHIVE.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        if ARCHIVE.exists():
            ARCHIVE.unlink()
        subprocess.run(["ar", "rcs", str(ARCHIVE), *map(str, objs)], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
