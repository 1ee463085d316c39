"""Generate the golden fixtures of the tile path from the reference's own code.

Runs in a container where the reference tree and oracle/_ref/libmf_refhost.so
(the reference's Tile_create + blockspmv_cpu compiled from its sources by
oracle/Makefile) exist:

    python tests/golden/make_golden.py

Writes tests/golden/tiles_small.npz (full input CSR and every reference-layout
array for small seeded matrices) and tests/golden/tiles_hashes.json (SHA-256 of
each array for the larger seeded systems).  Inputs are regenerated from their
seeds by millefeuille.matrices, and also stored for the small cases.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "mille-feuille_b200"))

import oracle  # noqa: E402
from millefeuille import matrices as M  # noqa: E402


def small_cases():
    """(name, rowA, colA, CSR) -- shapes chosen to hit the reference's corner cases."""
    yield "rand_unsorted", 192, 230, M.random_csr(200, 230, 0.05, seed=11, shuffle_cols=True, empty_rows=0.1)
    yield "rand_dense_tiles", 96, 96, M.random_csr(96, 96, 0.1, seed=12, dense_tile_rows=3)
    yield "rand_ragged_rows", 77, 77, M.random_csr(77, 77, 0.3, seed=13)
    yield "rand_wide", 64, 1000, M.random_csr(64, 1000, 0.02, seed=14, empty_rows=0.2)
    yield "empty_rows_only", 32, 32, M.random_csr(32, 32, 0.0, seed=15, empty_rows=1.0)
    yield "lap2d_32", 1024, 1024, M.laplace2d(32)
    A, _, _ = M.poisson3d_varcoef(8, seed=1)
    yield "poisson3d_8", A.n, A.n, A
    A, _, _ = M.convdiff3d(8, seed=2)
    yield "convdiff3d_8", A.n, A.n, A


def hash_cases():
    yield "lap2d_256", M.laplace2d(256)
    A, _, _ = M.poisson3d_varcoef(32, seed=1)
    yield "poisson3d_32", A
    A, _, _ = M.convdiff3d(24, seed=2)
    yield "convdiff3d_24", A


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libmf_refhost.so is missing: run `make -C oracle REF_SRC=<reference>/src`")
    out = {}
    for name, rowA, colA, A in small_cases():
        dims, arrs = oracle.ref_tile_create(rowA, colA, A.rowptr, A.colidx, A.val)
        out[f"{name}/in_rowptr"] = A.rowptr
        out[f"{name}/in_colidx"] = A.colidx
        out[f"{name}/in_val"] = A.val
        out[f"{name}/shape"] = np.array([rowA, colA], dtype=np.int64)
        for k, v in arrs.items():
            out[f"{name}/{k}"] = v
        print(name, dims)
    np.savez_compressed(os.path.join(HERE, "tiles_small.npz"), **out)
    hashes = {}
    for name, A in hash_cases():
        dims, arrs = oracle.ref_tile_create(A.n, A.n, A.rowptr, A.colidx, A.val)
        hashes[name] = {"dims": dims, "sha256": {k: sha(v) for k, v in arrs.items()}}
        print(name, dims)
    with open(os.path.join(HERE, "tiles_hashes.json"), "w") as f:
        json.dump(hashes, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
