"""Build libmillefeuille.so in-tree for sm_100a with nvcc (no JIT cache).

    python mille-feuille_b200/build.py [--verbose]

Object files go to mille-feuille_b200/_build/, the shared libraries to
mille-feuille_b200/millefeuille/: libmillefeuille.so (cg_solve_inc is the
mixed-precision solver of main-cg-mixed.cu) and libmillefeuille_fp64.so (the
same objects with api.cu built with MF_CG_INC_FP64: cg_solve_inc is the FP64
solver of main-cg.cu).  The drop-in driver executables (main-cg, main-cg-mixed,
main-bicg, main-bicg-mixed) go to mille-feuille_b200/bin/, main-cg linked
against the FP64 variant (all git-ignored, carried with the tree).  Rebuilds
only what changed.

    python mille-feuille_b200/build.py --check

also builds libmillefeuille_check.so: solver.cu and api.cu compiled with
MF_CHECK, every kernel index taken from stored data checked against its
array's extent (MF_ERR_CHECK on a failed check; the access is skipped).  Load
it with MILLEFEUILLE_LIB=<path> in place of libmillefeuille.so.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "millefeuille", "libmillefeuille.so")
OUT_FP64 = os.path.join(HERE, "millefeuille", "libmillefeuille_fp64.so")
OUT_CHECK = os.path.join(HERE, "millefeuille", "libmillefeuille_check.so")
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


def _compile(src: str, obj: str, deps, verbose: bool, defines=()) -> None:
    if not _newer(src, obj, deps):
        return
    cmd = [NVCC, *ARCH, *CUFLAGS, *[f"-D{d}" for d in defines], "-c", src, "-o", obj]
    if verbose and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    if src.endswith(".cpp"):
        cmd = ["g++", "-O2", "-fPIC", "-pthread", "-std=c++17", "-I", INCLUDE, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode:
        raise RuntimeError(f"compile failed: {os.path.basename(src)}")


def _link(out: str, objs) -> None:
    if any(_newer(o, out, []) for o in objs) or not os.path.exists(out):
        cmd = [NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart", "-Xcompiler", "-pthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"link failed: {os.path.basename(out)}")


def build(verbose: bool = False, check: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "millefeuille.h")]
    jobs, objs = [], []                  # (source, object, defines)
    for src in SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        jobs.append((src, obj, ()))
    api_fp64 = os.path.join(BUILD, "api_fp64.cu.o")
    jobs.append(("api.cu", api_fp64, ("MF_CG_INC_FP64",)))
    swap = {}
    if check:
        for src in ("solver.cu", "api.cu"):
            obj = os.path.join(BUILD, src.replace(".cu", "_check.cu.o"))
            swap[src + ".o"] = obj
            jobs.append((src, obj, ("MF_CHECK",)))
    # the translation units compile independently: one nvcc per core
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_compile, os.path.join(CSRC, src), obj, deps, verbose, d) for src, obj, d in jobs]:
            f.result()
    _link(OUT, objs)
    _link(OUT_FP64, [api_fp64 if o.endswith("api.cu.o") else o for o in objs])
    if check:
        _link(OUT_CHECK, [swap.get(os.path.basename(o), o) for o in objs])
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
        # main-cg replaces main-cg.cu, whose cg_solve_inc is FP64
        lib = OUT_FP64 if name == "main-cg" else OUT
        if not _newer(src, exe, [lib, os.path.join(INCLUDE, "millefeuille.h")]):
            continue
        cmd = ["g++", "-O2", "-std=c++17", f"-DMF_DRIVER={k}", "-I", INCLUDE, src, "-o", exe,
               "-L", os.path.dirname(OUT), "-l" + os.path.basename(lib)[3:-3], "-Wl,-rpath,$ORIGIN/../millefeuille"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"driver build failed: {name}")


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, check="--check" in sys.argv))
