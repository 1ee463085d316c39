"""GPU parity of the csr2block tiler and the precision encoder: every array the
GPU builds is compared bit for bit with the oracle restatement (itself pinned to
the reference's Tile_create by the golden fixtures) and with those fixtures."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

TILE_KEYS = ["tile_ptr", "tile_columnidx", "tile_nnz", "blknnz", "csr_offset", "csrptr_offset", "val", "val_low",
             "col", "ptr", "ptroffset1", "ptroffset2", "blkcoostylerowidx", "colstart", "colstop"]
LIST_KEYS = ["nonzero_row_new", "blockrowid_new", "blockcsr_ptr_new", "tile_rowidx", "block_signal"]


def _gpu_arrays(mf, A, keys):
    return {k: A.export(k) for k in keys}


def _check_against_oracle(mf, oracle_mod, rowA, colA, rowptr, colidx, val):
    G = mf.Matrix.from_csr(rowA, colA, rowptr, colidx, val)
    T = oracle_mod.Tiles(rowA, colA, rowptr, colidx, val)
    o = T.arrays()
    g = _gpu_arrays(mf, G, TILE_KEYS + LIST_KEYS)
    for k in TILE_KEYS + LIST_KEYS:
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)
    return G, T, g


def test_gpu_tiles_match_golden(mf, oracle_mod, cuda):
    z = np.load(os.path.join(GOLD, "tiles_small.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    for name in names:
        rowA, colA = (int(v) for v in z[f"{name}/shape"])
        G, T, g = _check_against_oracle(mf, oracle_mod, rowA, colA, z[f"{name}/in_rowptr"], z[f"{name}/in_colidx"],
                                        z[f"{name}/in_val"])
        for k in TILE_KEYS:
            np.testing.assert_array_equal(g[k], z[f"{name}/{k}"], err_msg=f"{name}:{k}")


def test_gpu_tiles_match_golden_hashes(mf, cuda):
    from millefeuille import matrices as M
    with open(os.path.join(GOLD, "tiles_hashes.json")) as f:
        H = json.load(f)
    mats = {"lap2d_256": M.laplace2d(256), "poisson3d_32": M.poisson3d_varcoef(32, seed=1)[0],
            "convdiff3d_24": M.convdiff3d(24, seed=2)[0]}
    for name, A in mats.items():
        G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
        for k, h in H[name]["sha256"].items():
            assert hashlib.sha256(np.ascontiguousarray(G.export(k)).tobytes()).hexdigest() == h, f"{name}:{k}"


@pytest.mark.parametrize("seed", range(8))
def test_gpu_tiles_random(mf, oracle_mod, cuda, seed):
    from millefeuille import matrices as M
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(1, 700))
    ncols = int(rng.integers(max(n, 1), n + 300))
    A = M.random_csr(n, ncols, float(rng.uniform(0.0, 0.15)), seed=seed, empty_rows=float(rng.uniform(0, 0.4)),
                     dense_tile_rows=int(rng.integers(0, 3)) if n >= 16 and ncols >= 16 else 0)
    rowA = int(rng.integers(0, n + 1))
    _check_against_oracle(mf, oracle_mod, rowA, ncols, A.rowptr, A.colidx, A.val)


def test_gpu_tiles_wide_span_global_scratch(mf, oracle_mod, cuda):
    """Tile-rows whose column-tile span is too wide for shared memory use the
    global-scratch path of the tiler; results are identical."""
    from millefeuille import matrices as M
    n, ncols = 64, 400000
    rng = np.random.default_rng(5)
    rows = [np.unique(rng.integers(0, ncols, size=40)) for _ in range(n)]
    rowptr = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.int32)
    colidx = np.concatenate(rows).astype(np.int32)
    colidx[::7] = ncols - 1 - colidx[::7]      # keep the span wide, order unsorted
    val = rng.standard_normal(colidx.size)
    _check_against_oracle(mf, oracle_mod, n, ncols, rowptr, colidx, val)


def test_gpu_tiles_from_device_pointers(mf, oracle_mod, cuda):
    import torch
    from millefeuille import matrices as M
    A, _, _ = M.poisson3d_varcoef(16, seed=1)
    G = mf.Matrix.from_csr(A.n, A.n, torch.from_numpy(A.rowptr).to(cuda), torch.from_numpy(A.colidx).to(cuda),
                           torch.from_numpy(A.val).to(cuda))
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val).arrays()
    for k in TILE_KEYS + LIST_KEYS:
        np.testing.assert_array_equal(G.export(k), T[k], err_msg=k)


def test_gpu_encoder_matches_oracle(mf, oracle_mod, cuda):
    from millefeuille import matrices as M
    A = M.random_csr(400, 400, 0.05, seed=9)
    rng = np.random.default_rng(2)
    A.val = A.val * 10.0 ** rng.uniform(-7, 7, A.val.size)
    A.val[::11] = np.round(A.val[::11])
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    a = T.arrays()
    f16, i8 = oracle_mod.encode_ref(a["val"], a["val_low"])
    np.testing.assert_array_equal(G.export("val_f16"), f16)
    np.testing.assert_array_equal(G.export("val_i8_ref"), i8)
    q, s = oracle_mod.encode_i8_scaled(T)
    np.testing.assert_array_equal(G.export("i8_scale"), s)
    np.testing.assert_array_equal(G.export("val_i8"), q)


def test_gpu_reference_labels_match_oracle(mf, oracle_mod, cuda):
    from millefeuille import _lib
    import ctypes as C
    rng = np.random.default_rng(3)
    nseg = 4000
    p_old = rng.standard_normal(nseg * 16)
    # per segment a scale around the thresholds 1e-5 .. 1e-8, exact threshold hits included
    scale = 10.0 ** rng.uniform(-9.5, -4.5, nseg)
    p_new = p_old + np.repeat(scale, 16) * rng.uniform(-1, 1, nseg * 16)
    p_new[:64] = p_old[:64] + np.array([1e-5, 1e-6, 1e-7, 1e-8] * 16)
    vis = np.zeros(nseg, dtype=np.int32)
    _lib.check(_lib.load().mf_debug_ref_labels(p_old.ctypes.data_as(C.c_void_p), p_new.ctypes.data_as(C.c_void_p),
                                                nseg, vis.ctypes.data_as(C.c_void_p), 0))
    np.testing.assert_array_equal(vis, oracle_mod.segment_labels_ref(p_old, p_new))
    assert set(np.unique(vis)) == {0, 1, 2, 3, 4}
