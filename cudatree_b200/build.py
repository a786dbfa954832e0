"""Build libcudatree_b200.so for sm_100a with nvcc (in-tree, no JIT cache).

Usage: ``python -m cudatree_b200.build [--force] [--ptxas-verbose]``.
Objects go to ``cudatree_b200/_build``; the shared library is written next
to this file so that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libcudatree_b200.so"
INCLUDE = HERE.parent / "include"

SOURCES = [
    "ct_api.cu",
    "ct_level.cu",
    "ct_fit.cu",
    "ct_boot.cu",
    "ct_predict.cu",
    "ct_presort.cu",
    "ct_partition.cu",
    "ct_noalloc.cu",
    "ct_server.cu",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wall", "-I", str(INCLUDE)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu*")) + sorted(INCLUDE.glob("*.h")) + [Path(__file__)]


def _compile(src: Path, ptxas_verbose: bool) -> tuple[Path, str]:
    obj = BUILD / (src.stem + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True) -> Path:
    """Compile every kernel source and link the shared library; return its path."""
    srcs = [CSRC / s for s in SOURCES]
    if not force and LIB.exists():
        newest = max(p.stat().st_mtime for p in _deps())
        if LIB.stat().st_mtime >= newest:
            return LIB
    BUILD.mkdir(exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_verbose), srcs))
    if ptxas_verbose:
        for _, log in results:
            sys.stderr.write(log)
    objs = [str(o) for o, _ in results]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    if not quiet:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    args = ap.parse_args()
    build(force=args.force, ptxas_verbose=args.ptxas_verbose, quiet=False)
