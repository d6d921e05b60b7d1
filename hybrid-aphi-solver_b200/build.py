"""Builds libaphi_b200.so in-tree for sm_100a with nvcc.

    python hybrid-aphi-solver_b200/build.py [--force] [-j N]

Objects go to hybrid-aphi-solver_b200/_build/, the library to
hybrid-aphi-solver_b200/aphi_b200/libaphi_b200.so, where the Python package
loads it. Rebuilds only what changed (source or any header newer than the
object).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = PKG / "aphi_b200" / "libaphi_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2,-pthread",
          f"-I{ROOT / 'include'}", f"-I{CSRC}"]
# Element fill and scatter reproduce the host's rounding: no FMA contraction.
PER_FILE = {
    "assembly.cu": ["-fmad=false"],
    "csc_solve.cu": ["-fmad=false"],
}


def sources():
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp"))


def headers():
    return [p for p in list(CSRC.iterdir()) + list((ROOT / "include").iterdir())
            if p.suffix in (".h", ".hpp", ".cuh")]


def compile_one(src: Path, force: bool) -> Path:
    obj = OUT / (src.name + ".o")
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in headers()]
                 + [Path(__file__).stat().st_mtime])
    if not force and obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [NVCC, *ARCH, *COMMON, *PER_FILE.get(src.name, []), "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, jobs: int = 8, verbose: bool = True) -> Path:
    OUT.mkdir(exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force), srcs))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcuda", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    build(a.force, a.j)
