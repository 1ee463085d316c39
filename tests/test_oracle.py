"""CPU tests: the oracle restatement against the reference's own host code
(golden fixtures made by tests/golden/make_golden.py from Tile_create /
blockspmv_cpu compiled from the reference sources), and its solvers against
direct solves."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _golden_cases():
    z = np.load(os.path.join(GOLD, "tiles_small.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    return z, names


REF_KEYS = ["tile_ptr", "tile_columnidx", "tile_nnz", "blknnz", "csr_offset", "csrptr_offset", "val",
            "val_low", "col", "ptr", "ptroffset1", "ptroffset2", "blkcoostylerowidx", "colstart", "colstop"]


@pytest.mark.parametrize("case", _golden_cases()[1])
def test_oracle_tiles_match_reference_golden(oracle_mod, case):
    z, _ = _golden_cases()
    rowA, colA = (int(v) for v in z[f"{case}/shape"])
    T = oracle_mod.Tiles(rowA, colA, z[f"{case}/in_rowptr"], z[f"{case}/in_colidx"], z[f"{case}/in_val"])
    a = T.arrays()
    for k in REF_KEYS:
        np.testing.assert_array_equal(a[k], z[f"{case}/{k}"], err_msg=f"{case}:{k}")


def test_oracle_tiles_match_reference_hashes(oracle_mod):
    import hashlib
    from millefeuille import matrices as M
    with open(os.path.join(GOLD, "tiles_hashes.json")) as f:
        H = json.load(f)
    mats = {"lap2d_256": M.laplace2d(256), "poisson3d_32": M.poisson3d_varcoef(32, seed=1)[0],
            "convdiff3d_24": M.convdiff3d(24, seed=2)[0]}
    for name, A in mats.items():
        T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
        a = T.arrays()
        for k, h in H[name]["sha256"].items():
            assert hashlib.sha256(np.ascontiguousarray(a[k]).tobytes()).hexdigest() == h, f"{name}:{k}"


@pytest.mark.parametrize("seed", range(6))
def test_oracle_tiles_match_reference_live(oracle_mod, seed):
    """Random shapes against the reference compiled in oracle/_ref (when built here)."""
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built")
    from millefeuille import matrices as M
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(17, 300))
    ncols = int(rng.integers(n, n + 80))
    A = M.random_csr(n, ncols, float(rng.uniform(0.005, 0.2)), seed=seed, empty_rows=0.15,
                     dense_tile_rows=int(rng.integers(0, 3)))
    rowA = int(rng.integers(1, n + 1))
    dims, ref = oracle_mod.ref_tile_create(rowA, ncols, A.rowptr, A.colidx, A.val)
    a = oracle_mod.Tiles(rowA, ncols, A.rowptr, A.colidx, A.val).arrays()
    for k in REF_KEYS:
        np.testing.assert_array_equal(a[k], ref[k], err_msg=k)


def test_rowlists_consistent_with_tiles(oracle_mod):
    """The nonempty-row lists (main-cg-mixed.cu:2447-2514) reproduce the tile
    SpMV exactly when no tile holds 256 entries (uint8 end offsets do not wrap)."""
    from millefeuille import matrices as M
    A = M.random_csr(300, 300, 0.05, seed=3, empty_rows=0.1)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    x = np.random.default_rng(0).standard_normal(A.n)
    np.testing.assert_allclose(T.spmv_tile(x), A.to_scipy() @ x, rtol=1e-13, atol=1e-13)


def test_rowlists_dense_tile_wrap_is_reference_behaviour(oracle_mod):
    """A 256-entry tile's last row end offset wraps to 0 in the reference's
    uint8 lists, so its verification loop drops that row; the restatement keeps
    that behaviour (parity), the solvers use exact offsets."""
    from millefeuille import matrices as M
    A = M.random_csr(32, 32, 0.0, seed=4, empty_rows=1.0, dense_tile_rows=1)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    a = T.arrays()
    assert 0 in a["blockcsr_ptr_new"][1:]
    x = np.ones(A.n)
    y_ref = A.to_scipy() @ x
    y = T.spmv_tile(x)
    assert np.any(np.abs(y - y_ref) > 1e-9)


def test_encoder_half_rounding_matches_ieee(oracle_mod):
    rng = np.random.default_rng(7)
    v = np.concatenate([rng.standard_normal(20000) * 10 ** rng.uniform(-9, 6, 20000),
                        [0.0, -0.0, 65504.0, 65520.0, 1e6, 6e-8, 5.96e-8, 2.98e-8, np.inf, -np.inf]])
    f32 = v.astype(np.float32)
    f16, i8 = oracle_mod.encode_ref(v, f32)
    with np.errstate(over="ignore"):     # values past FP16's range round to inf on purpose
        want = f32.astype(np.float16).view(np.uint16)
    np.testing.assert_array_equal(f16, want)
    w = np.trunc(v[np.isfinite(v) & (np.abs(v) < 2 ** 31)]).astype(np.int64)
    np.testing.assert_array_equal(i8[: w.size][np.abs(v[: w.size]) < 2 ** 31],
                                  (w & 0xFF).astype(np.uint8).view(np.int8)[np.abs(v[: w.size]) < 2 ** 31])


def test_label_classification_table(oracle_mod):
    # main-cg-mixed.cu:1334-1369: thresholds 1e-5, 1e-6, 1e-7, 1e-8
    lib = oracle_mod.lib()
    cases = {2e-5: 1, 1e-5: 4, 5e-6: 4, 1e-6: 3, 5e-7: 3, 1e-7: 2, 5e-8: 2, 1e-8: 0, 0.0: 0, float("nan"): 0}
    for dp, code in cases.items():
        assert lib.orc_classify_ref(dp) == code, dp
    p0 = np.zeros(64)
    p1 = np.zeros(64)
    p1[3] = 2e-5          # segment 0 -> fp64
    p1[20] = 5e-7         # segment 1 -> fp16
    p1[21] = 5e-6         # ... and fp32: most conservative wins
    p1[40] = 5e-8         # segment 2 -> int8
    assert list(oracle_mod.segment_labels_ref(p0, p1)) == [0, 4, 2, 1]


def test_oracle_cg_matches_direct_solve(oracle_mod):
    from millefeuille import matrices as M
    A, b, xt = M.laplace2d_system(24, seed=0)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = T.cg_fp64(b, tol=1e-12, max_iter=5000)
    assert rep["converged"] and rep["relres_true"] <= 1e-12
    import scipy.sparse.linalg as sla
    xd = sla.spsolve(A.to_scipy().tocsc(), b)
    np.testing.assert_allclose(x, xd, rtol=0, atol=1e-9)


def test_oracle_bicgstab_matches_direct_solve(oracle_mod):
    from millefeuille import matrices as M
    A, b, _ = M.convdiff3d(12, seed=2)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = T.bicgstab_fp64(b, tol=1e-12, max_iter=5000)
    assert rep["converged"] and rep["relres_true"] <= 1e-12
    import scipy.sparse.linalg as sla
    xd = sla.spsolve(A.to_scipy().tocsc(), b)
    np.testing.assert_allclose(x, xd, rtol=1e-8, atol=1e-10)


def test_oracle_fixed_iterations(oracle_mod):
    from millefeuille import matrices as M
    A, b, _ = M.poisson3d_varcoef(8, seed=1)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    _, rep = T.cg_fp64(b, tol=1e-30, max_iter=17, fixed_iters=True)
    assert rep["iterations"] == 17 and not rep["converged"]


def test_generators_shapes():
    from millefeuille import matrices as M
    A = M.laplace2d(256)
    assert A.n == 65536 and A.nnz == 326656
    A, b, xt = M.poisson3d_varcoef(16, seed=1)
    assert A.n == 4096 and A.nnz == 7 * 4096 - 6 * 16 * 16
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0
    d = S.diagonal()
    off = np.asarray(abs(S).sum(axis=1)).ravel() - d
    assert np.all(d >= off * (1 - 1e-14)) and np.any(d > off)   # weakly dominant, strictly on the boundary
    A, b, pe = M.convdiff3d(16, seed=2)
    assert A.n == 4096 and pe == pytest.approx(10 * (2 * np.pi / 16) / 2, rel=0.03)  # max sin at cell centres < 1


def test_batch_systems_generator():
    """The batched workload: seeded kinds / sides / right-hand-side counts,
    SPD 5-point and 27-point systems."""
    from millefeuille import matrices as M
    sy = M.batch_systems(8, seed=3, side2d=(6, 30), side3d=(3, 9), rhs=(1, 16))
    sy2 = M.batch_systems(8, seed=3, side2d=(6, 30), side3d=(3, 9), rhs=(1, 16))
    for (kind, side, A, B), (k2, s2, A2, B2) in zip(sy, sy2):
        assert (kind, side) == (k2, s2) and np.array_equal(A.val, A2.val) and np.array_equal(B, B2)
        n = side ** (2 if kind == "2d5" else 3)
        assert A.n == n and B.shape[1] == n and 1 <= B.shape[0] <= 16
        S = A.to_scipy()
        assert abs(S - S.T).max() == 0
        assert np.diff(A.rowptr).max() == (5 if kind == "2d5" else 27)
        assert np.linalg.eigvalsh(S.toarray()).min() > 0


def test_aniso2d_grf_generator():
    """The differentiable-solve workload: SPD 5-point system, GRF of unit
    variance, x-couplings ratio times the y-couplings, seeded."""
    from millefeuille import matrices as M
    A, B, Xt, kap = M.aniso2d_grf(64, seed=4, corr=16.0, nrhs=3)
    assert A.n == 4096 and A.nnz == 5 * 4096 - 4 * 64 and B.shape == (3, 4096) and Xt.shape == (3, 4096)
    g = np.log(kap)
    assert abs(g.mean()) < 1e-12 and g.std() == pytest.approx(1.0, rel=1e-12)
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0
    d = S.diagonal()
    off = np.asarray(abs(S).sum(axis=1)).ravel() - d
    assert np.all(d >= off * (1 - 1e-14)) and np.any(d > off)
    # interior cell 65 (x=1, y=1): x-coupling = 10 * harmonic mean of kappa, y-coupling = harmonic mean
    hm = lambda a, b: 2 * a * b / (a + b)
    assert S[65, 66] == pytest.approx(-10 * hm(kap[1, 1], kap[1, 2]), rel=1e-14)
    assert S[65, 129] == pytest.approx(-hm(kap[1, 1], kap[2, 1]), rel=1e-14)
    A2, B2, _, _ = M.aniso2d_grf(64, seed=4, corr=16.0, nrhs=3)
    assert np.array_equal(A2.val, A.val) and np.array_equal(B2, B)


def test_oracle_f64_to_f16_and_hfma(oracle_mod):
    """The oracle's binary16 conversion matches numpy's (round to nearest even
    from binary64, overflow to inf, subnormals); __hfma's single rounding is
    checked against the exact rational a*b + c rounded to the nearest half."""
    from fractions import Fraction
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.standard_normal(20000) * 10.0 ** rng.integers(-9, 6, 20000),
                        [65504.0, 65519.99, 65520.0, 6e-8, 2.98e-8, 2.0 ** -25, -0.0, 0.0, np.inf, -np.inf]])
    with np.errstate(over="ignore"):
        ref = v.astype(np.float16).view(np.uint16)
    got = np.array([oracle_mod.f64_to_f16_rn(t) for t in v], dtype=np.uint16)
    np.testing.assert_array_equal(got, ref)
    # a tie of s alone broken by the error term: 1 + 2^-11 is halfway between 1 and 1 + 2^-10
    s = 1.0 + 2.0 ** -11
    assert oracle_mod.f64_to_f16_rn(s, 0.0) == 0x3C00             # ties to even -> 1.0
    assert oracle_mod.f64_to_f16_rn(s, 2.0 ** -60) == 0x3C01      # just above the tie
    assert oracle_mod.f64_to_f16_rn(-s, -(2.0 ** -60)) == 0xBC01  # magnitude above the tie

    def h2f(h):
        return Fraction(float(np.array([h], dtype=np.uint16).view(np.float16)[0]))

    def nearest(fr):
        f = float(fr)
        base = int(np.array([np.float16(f)]).view(np.uint16)[0])
        best = None
        for d in (-2, -1, 0, 1, 2):
            c = (base + d) & 0xFFFF
            val = np.array([c], dtype=np.uint16).view(np.float16)[0]
            if not np.isfinite(val):
                continue
            key = (abs(Fraction(float(val)) - fr), c & 1)
            if best is None or key < best[0]:
                best = (key, c)
        return best[1]

    for _ in range(3000):
        a, b, c = (np.float16(rng.standard_normal() * 10.0 ** rng.integers(-4, 3)) for _ in range(3))
        ha, hb, hc = (int(np.array([t]).view(np.uint16)[0]) for t in (a, b, c))
        exact = h2f(ha) * h2f(hb) + h2f(hc)
        if exact == 0 or abs(float(exact)) > 60000:
            continue
        assert oracle_mod.hfma(ha, hb, hc) == nearest(exact)


def test_oracle_spmv_slices_and_parity_cg(oracle_mod):
    """The slice-order product of the encoded values agrees with the FP64 CSR
    product within each encoding's rounding; with every label FP64 (b of unit
    size, so |p_new - p_old| > 1e-5 everywhere) the parity-mode CG is the FP64
    CG of the same schedule."""
    from millefeuille import matrices as M
    A = M.random_csr(200, 230, 0.08, seed=4)
    T = oracle_mod.Tiles(A.n, 230, A.rowptr, A.colidx, A.val)
    x = np.random.default_rng(1).uniform(-1, 1, 230)
    import scipy.sparse as sp
    S = sp.csr_matrix((A.val, A.colidx, A.rowptr), shape=(A.n, 230))
    ye, sc = S @ x, abs(S) @ np.abs(x)
    for prec, rel in ((0, 1e-14), (1, 1.2e-7), (2, 1e-3)):
        assert np.all(np.abs(T.spmv_slices(x, prec) - ye) <= rel * sc)
    A2, b2, _ = M.laplace2d_system(24, seed=0)
    T2 = oracle_mod.Tiles(A2.n, A2.n, A2.rowptr, A2.colidx, A2.val)
    for k in (1, 5, 12):
        xp, lab, agree, rp = T2.cg_parity(b2, k)
        xf, rf = T2.cg_fp64(b2, max_iter=k, fixed_iters=True)
        assert np.all(lab == 0)
        np.testing.assert_allclose(xp, xf, rtol=1e-10, atol=1e-12 * np.abs(xf).max())
        assert rp["relres_true"] == pytest.approx(rf["relres_true"], rel=1e-8)
    # scaled right-hand side: labels spread over the reduced classes, deterministically
    xa, la, _, _ = T2.cg_parity(b2 * 2e-6, 20)
    xb, lb, _, _ = T2.cg_parity(b2 * 2e-6, 20)
    np.testing.assert_array_equal(la, lb)
    np.testing.assert_array_equal(xa, xb)
    assert set(la.tolist()) >= {2, 3}
