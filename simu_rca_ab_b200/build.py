"""Builds librcabf.so in-tree for sm_100a.

    python -m simu_rca_ab_b200.build            # incremental
    python -m simu_rca_ab_b200.build --clean

Every CUDA translation unit is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a``; the host C++ units with the
system g++.  The translation units holding the reference-compatible
arithmetic are compiled with ``-fmad=false`` so that no multiply is fused
into a following add.  Objects go to ``simu_rca_ab_b200/_build/``; the
library is written next to this file, where the Python binding loads it.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "librcabf.so"

NVCC = os.environ.get("RCABF_NVCC", "nvcc")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
HOST_CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                     "-ccbin", HOST_CXX, "-I", str(CSRC), "-I", str(INCLUDE)]
# reference-compatible arithmetic: no FMA contraction
STRICT_UNITS = {"fused_ref.cu", "tables_ref.cu"}
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
             "-I", str(CSRC), "-I", str(INCLUDE), "-I", f"{CUDA_HOME}/include"]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, verbose: bool) -> tuple[Path, str]:
    obj = BUILD / (src.name + ".o")
    if src.suffix == ".cu":
        cmd = [NVCC] + NVCC_FLAGS + (["-fmad=false"] if src.name in STRICT_UNITS else [])
        cmd += ["-c", str(src), "-o", str(obj)]
    else:
        cmd = [HOST_CXX] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(clean: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compiles the CUDA/C++ sources (incrementally) and links librcabf.so."""
    if clean and BUILD.exists():
        shutil.rmtree(BUILD)
    BUILD.mkdir(exist_ok=True)
    hdr = _headers_mtime()
    todo = []
    objs = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr):
            todo.append(src)
    if todo:
        jobs = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for obj, err in ex.map(lambda s: _compile(s, verbose), todo):
                if verbose and err.strip():
                    print(err, file=sys.stderr)
    newest = max(o.stat().st_mtime for o in objs)
    if todo or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX, "-o", str(tmp)]
        cmd += [str(o) for o in objs] + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=None)
    a = ap.parse_args()
    print(build(a.clean, a.verbose, a.jobs))


if __name__ == "__main__":
    main()
