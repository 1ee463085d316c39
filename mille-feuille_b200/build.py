"""Build libmillefeuille.so in-tree for sm_100a with nvcc (no JIT cache).

    python mille-feuille_b200/build.py [--verbose]

Object files go to mille-feuille_b200/_build/, the shared library to
mille-feuille_b200/millefeuille/libmillefeuille.so (git-ignored, carried with
the tree).  Rebuilds only what changed.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "millefeuille", "libmillefeuille.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-ccbin", "g++", "-I", INCLUDE]
SOURCES = ["scan.cu", "tile_build.cu", "solver.cu", "api.cu", "adjoint.cu", "mmio.cpp"]
HEADERS = ["mf_internal.cuh"]


def _newer(src: str, dst: str, deps) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in [src, *deps])


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "millefeuille.h")]
    objs = []
    for src in SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not _newer(sp, obj, deps):
            continue
        cmd = [NVCC, *ARCH, *CUFLAGS, "-c", sp, "-o", obj]
        if verbose and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cpp"):
            cmd = ["g++", "-O2", "-fPIC", "-std=c++17", "-I", INCLUDE, "-c", sp, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"compile failed: {src}")
    if any(_newer(o, OUT, []) for o in objs) or not os.path.exists(OUT):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
