"""Build libmillefeuille.so in-tree for sm_100a with nvcc (no JIT cache).

    python mille-feuille_b200/build.py [--verbose]

Object files go to mille-feuille_b200/_build/, the shared library to
mille-feuille_b200/millefeuille/libmillefeuille.so and the drop-in driver
executables (main-cg, main-cg-mixed, main-bicg, main-bicg-mixed) to
mille-feuille_b200/bin/ (all git-ignored, carried with the tree).  Rebuilds
only what changed.
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
            cmd = ["g++", "-O2", "-fPIC", "-pthread", "-std=c++17", "-I", INCLUDE, "-c", sp, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"compile failed: {src}")
    if any(_newer(o, OUT, []) for o in objs) or not os.path.exists(OUT):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart", "-Xcompiler", "-pthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    build_drivers(verbose)
    return OUT


DRIVERS = ["main-cg", "main-cg-mixed", "main-bicg", "main-bicg-mixed"]
BIN = os.path.join(HERE, "bin")


def build_drivers(verbose: bool = False) -> None:
    """The reference's four benchmark executables over the library
    (csrc/driver_main.cpp, variant chosen by MF_DRIVER) into bin/."""
    os.makedirs(BIN, exist_ok=True)
    src = os.path.join(CSRC, "driver_main.cpp")
    for k, name in enumerate(DRIVERS):
        exe = os.path.join(BIN, name)
        if not _newer(src, exe, [OUT, os.path.join(INCLUDE, "millefeuille.h")]):
            continue
        cmd = ["g++", "-O2", "-std=c++17", f"-DMF_DRIVER={k}", "-I", INCLUDE, src, "-o", exe,
               "-L", os.path.dirname(OUT), "-lmillefeuille", "-Wl,-rpath,$ORIGIN/../millefeuille"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"driver build failed: {name}")


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
