"""GPU parity of the tile SpMV and the persistent CG / BiCGSTAB kernel against
the FP64 oracle (the reference's algorithm restated on the CPU).

Tolerances: SpMV FP64 rtol 1e-13 (summation order differs from the oracle's);
FP32 tiles rtol 1e-5; solver iteration counts within 5 % (+1) of the oracle's;
every converged solve is checked with an independent FP64 residual."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _relres(A, x, b):
    return np.linalg.norm(A.to_scipy() @ x - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def lap64():
    from millefeuille import matrices as M
    return M.laplace2d_system(64, seed=0)


@pytest.fixture(scope="module")
def p3d():
    from millefeuille import matrices as M
    return M.poisson3d_varcoef(32, seed=1)


@pytest.fixture(scope="module")
def cd3d():
    from millefeuille import matrices as M
    return M.convdiff3d(20, seed=2)


def test_gpu_spmv_fp64_and_fp32(mf, cuda):
    from millefeuille import matrices as M
    for A in (M.laplace2d(64), M.poisson3d_varcoef(24, seed=1)[0], M.random_csr(500, 530, 0.03, seed=2)):
        ncols = int(A.colidx.max()) + 1 if A.nnz else A.n
        ncols = max(ncols, A.n)
        G = mf.Matrix.from_csr(A.n, ncols, A.rowptr, A.colidx, A.val)
        x = np.random.default_rng(0).standard_normal(ncols)
        S = A.to_scipy() if ncols == A.n else __import__("scipy.sparse", fromlist=["csr_matrix"]).csr_matrix(
            (A.val, A.colidx, A.rowptr), shape=(A.n, ncols))
        y_ref = S @ x
        y = G.spmv(x, precision="fp64")
        np.testing.assert_allclose(y, y_ref, rtol=1e-13, atol=1e-13 * np.abs(y_ref).max())
        y32 = G.spmv(x, precision="mixed")
        np.testing.assert_allclose(y32, y_ref, rtol=1e-5, atol=1e-5 * np.abs(y_ref).max())


def test_gpu_cg_fp64_matches_oracle(mf, oracle_mod, cuda, lap64):
    A, b, xt = lap64
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = G.solve(b, method="cg", precision="fp64", tol=1e-10, replace_every=0)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    xo, ro = T.cg_fp64(b, tol=1e-10, max_iter=10000)
    assert rep["converged"] and rep["relres_true"] <= 1e-10
    assert abs(rep["iterations"] - ro["iterations"]) <= 1 + 0.05 * ro["iterations"]
    assert _relres(A, x, b) <= 1e-10
    np.testing.assert_allclose(x, xo, rtol=0, atol=1e-7)
    assert np.abs(x - xt).max() < 1e-6


def test_gpu_cg_fp64_fixed_iterations_track_oracle(mf, oracle_mod, cuda, p3d):
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    # FP64 CG iterates of this system are rounding-sensitive: two summation
    # orders stay within 1e-13 for ~15 iterations, then drift apart (2e-7 at 30).
    for k in (1, 7, 15):
        x, rep = G.solve(b, precision="fp64", max_iter=k, fixed_iters=1, replace_every=0)
        xo, ro = T.cg_fp64(b, max_iter=k, fixed_iters=True)
        assert rep["iterations"] == k
        np.testing.assert_allclose(x, xo, rtol=1e-9, atol=1e-11 * np.abs(xo).max())
        assert rep["relres_true"] == pytest.approx(ro["relres_true"], rel=1e-6)


def test_gpu_cg_mixed_converges_fp64_verified(mf, oracle_mod, cuda, p3d):
    A, b, xt = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = G.solve(b, method="cg", precision="mixed", tol=1e-8)
    assert rep["converged"] and rep["relres_true"] <= 1e-8
    assert _relres(A, x, b) <= 1.0001e-8
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    _, ro = T.cg_fp64(b, tol=1e-8, max_iter=10000)
    # FP32-stored values cost a few iterations (measured 294 against 280 on this
    # 32^3 system, 1,509 against 1,402 on 128^3)
    assert rep["iterations"] <= 1.08 * ro["iterations"] + 3, (rep["iterations"], ro["iterations"])
    assert sum(rep["tile_uses"][1:]) > 0          # low-precision tiles were used


def test_gpu_mixed_usage_counters_cover_every_entry(mf, cuda, p3d):
    """The report's per-precision counters.  With every tile in FP32 (smooth
    right-hand side, no tile exact in a narrower type), each mixed-mode SpMV
    counts every tile and every stored entry once: the lean FP32 walk, which
    reads no row lengths, takes its entry count from the CSR row pointers of
    its tile-rows, and the totals must equal (SpMVs) x (tiles, nnz)."""
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = G.solve(b, method="cg", precision="mixed", tol=1e-8)
    T = G.info["tilenum"]
    tu, nu = rep["tile_uses"], rep["nnz_uses"]
    assert tu[0] == tu[2] == tu[3] == 0 and nu[0] == nu[2] == nu[3] == 0, (tu, nu)
    assert tu[1] % T == 0, (tu, T)
    nspmv = tu[1] // T
    assert nspmv >= rep["iterations"]
    assert nu[1] == nspmv * A.nnz, (nu, nspmv, A.nnz)


def test_gpu_mixed_demotes_small_segments_and_converges(mf, cuda, p3d):
    """A right-hand side confined to a few planes: most column segments of the
    SpMV operand are tiny or zero next to the largest, so their tiles run in
    FP16 / INT8; the solve still converges on the FP64 true residual.  A
    uniform right-hand side of the same system keeps every tile in FP32."""
    A, _, _ = p3d
    b = np.zeros(A.n)
    b[:3 * 32 * 32] = np.random.default_rng(3).standard_normal(3 * 32 * 32)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = G.solve(b, method="cg", precision="mixed", tol=1e-8)
    assert rep["converged"] and _relres(A, x, b) <= 1.0001e-8
    assert rep["tile_uses"][2] + rep["tile_uses"][3] > 0, rep["tile_uses"]
    # every SpMV counts each tile and each stored entry once, in the precision it ran
    T = G.info["tilenum"]
    assert sum(rep["tile_uses"]) % T == 0
    assert sum(rep["nnz_uses"]) == sum(rep["tile_uses"]) // T * A.nnz, (rep["tile_uses"], rep["nnz_uses"])
    # demote_min_fraction = 1: narrower tiles only if every segment is small -> all FP32
    x1, rep1 = G.solve(b, method="cg", precision="mixed", tol=1e-8, demote_min_fraction=1.0)
    assert rep1["converged"] and _relres(A, x1, b) <= 1.0001e-8
    assert rep1["tile_uses"][2] + rep1["tile_uses"][3] == 0 and rep1["tile_uses"][1] > 0, rep1["tile_uses"]
    X, reps = G.solve_multi(np.stack([b, b[::-1].copy()]), method="cg", precision="mixed", tol=1e-8)
    for k in range(2):
        assert reps[k]["converged"] and _relres(A, X[k], [b, b[::-1]][k]) <= 1.0001e-8


def test_gpu_mixed_converges_past_the_fp32_floor(mf, cuda):
    """A small well-conditioned 27-point system whose solve reaches the FP32
    products' accuracy floor (~1e-7) early: the recursive residual collapses
    below the true one, and the FP64 replacement must restart the direction
    instead of scaling it by r_true.r_true / r_old.r_old (which broke down).
    Single-column and multi-column kernels, CG; BiCGSTAB on the same system."""
    from millefeuille import matrices as M
    kind, side, A, B = M.batch_systems(14, seed=3, side2d=(8, 48), side3d=(4, 12), rhs=(1, 16))[0]
    assert kind == "3d27" and A.n == 125
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    for method in ("cg", "bicgstab"):
        x, rep = G.solve(B[0], method=method, precision="mixed", tol=1e-8)
        assert rep["converged"] and rep["relres_true"] <= 1e-8 and rep["iterations"] < 500, (method, rep)
        assert _relres(A, x, B[0]) <= 1.0001e-8
    X, reps = G.solve_multi(B, method="cg", precision="mixed", tol=1e-8)
    for k in range(B.shape[0]):
        assert reps[k]["converged"] and reps[k]["iterations"] < 500 and _relres(A, X[k], B[k]) <= 1.0001e-8


def test_gpu_cg_deterministic(mf, cuda, p3d):
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x1, r1 = G.solve(b, precision="mixed", tol=1e-8)
    x2, r2 = G.solve(b, precision="mixed", tol=1e-8)
    assert r1["iterations"] == r2["iterations"]
    np.testing.assert_array_equal(x1, x2)


def test_gpu_bicgstab_fp64_matches_oracle(mf, oracle_mod, cuda, cd3d):
    A, b, _ = cd3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = G.solve(b, method="bicgstab", precision="fp64", tol=1e-8, replace_every=0)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    xo, ro = T.bicgstab_fp64(b, tol=1e-8, max_iter=10000)
    assert rep["converged"] and rep["relres_true"] <= 1e-8
    assert abs(rep["iterations"] - ro["iterations"]) <= 2 + 0.05 * ro["iterations"]
    assert _relres(A, x, b) <= 1.0001e-8


def test_gpu_bicgstab_mixed_converges(mf, cuda, cd3d):
    A, b, _ = cd3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = G.solve(b, method="bicgstab", precision="mixed", tol=1e-8)
    assert rep["converged"] and rep["relres_true"] <= 1e-8
    assert _relres(A, x, b) <= 1.0001e-8


def test_gpu_solve_device_pointers(mf, cuda, p3d):
    import torch
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    bd = torch.from_numpy(b).to(cuda)
    xd, rep = G.solve(bd, precision="fp64", tol=1e-9)
    xh, rep2 = G.solve(b, precision="fp64", tol=1e-9)
    np.testing.assert_array_equal(xd.cpu().numpy(), xh)


def test_gpu_barrier_timeout_is_reported_and_context_survives(mf, cuda, lap64):
    A, b, _ = lap64
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    with pytest.raises(mf.MFError) as e:
        G.solve(b, precision="fp64", tol=1e-8, test_stall_barrier=1, wait_timeout_s=0.2)
    assert e.value.status == 4          # MF_ERR_TIMEOUT
    x, rep = G.solve(b, precision="fp64", tol=1e-8)
    assert rep["converged"]


def test_gpu_dropin_cg_solve_entry_points(mf, oracle_mod, cuda, p3d, tmp_path, monkeypatch):
    """cg_solve_sync / cg_solve_inc with the reference's argument list: exactly
    max_iter iterations, x returned, l2_norm = ||Ax-b||/||b|| in FP64."""
    from millefeuille import _lib
    monkeypatch.chdir(tmp_path)
    A, b, _ = p3d
    L = _lib.load()
    rp = A.rowptr.astype(np.int32).copy()
    ci = A.colidx.astype(np.int32).copy()
    vv = A.val.copy()
    vl = vv.astype(np.float32)
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    for name, prec in (("cg_solve_sync", "fp64"), ("cg_solve_inc", "mixed")):
        x = np.ones(A.n)
        res = _lib.CgBenchResult()
        it = C.c_int(0)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        getattr(L, name)(ip(rp), ip(ci), dp(vv), vl.ctypes.data_as(C.POINTER(C.c_float)), dp(x), dp(b.copy()),
                         A.n, C.byref(it), 10, 1e-5, b"p3d", A.nnz, A.n, 12, C.byref(res), 0)
        assert res.iterations == 12
        assert res.l2_norm == pytest.approx(_relres(A, x, b), rel=1e-6)
        if prec == "fp64":
            _, ro = T.cg_fp64(b, max_iter=12, fixed_iters=True)
            assert res.l2_norm == pytest.approx(ro["relres_true"], rel=1e-6)
    assert (tmp_path / "cg_performance.csv").exists() and (tmp_path / "cg_mixed_performance.csv").exists()


def test_gpu_dropin_bicgstab(mf, cuda, cd3d, tmp_path, monkeypatch):
    from millefeuille import _lib
    monkeypatch.chdir(tmp_path)
    A, _, _ = cd3d
    L = _lib.load()
    rhs = np.zeros(A.n)
    x = np.zeros(A.n)
    rc = L.bicgstab_sync(A.rowptr.ctypes.data_as(C.POINTER(C.c_int)), A.colidx.ctypes.data_as(C.POINTER(C.c_int)),
                         A.val.ctypes.data_as(C.POINTER(C.c_double)), rhs.ctypes.data_as(C.POINTER(C.c_double)),
                         x.ctypes.data_as(C.POINTER(C.c_double)), A.nnz, b"cd", A.n)
    assert rc == 0
    np.testing.assert_allclose(rhs, A.to_scipy() @ np.ones(A.n), rtol=1e-14)
    assert _relres(A, x, rhs) < 1e-6          # 50 fixed iterations on a well-conditioned system


@pytest.mark.parametrize("method,precision", [("cg", "fp64"), ("cg", "mixed"), ("bicgstab", "fp64"),
                                              ("bicgstab", "mixed")])
def test_gpu_ragged_system_with_decoupled_rows(mf, oracle_mod, cuda, method, precision):
    """A system whose size is not a multiple of 16 (the last tile-row is
    partial) and whose last 40 rows are decoupled, diagonal-only (tiles holding
    one entry per row): every method and precision converges on its FP64 true
    residual, and the FP64 CG agrees with the oracle's CG."""
    from millefeuille import matrices as M
    import scipy.sparse as sp
    L = M.laplace2d(31).to_scipy()                          # n = 961
    D = sp.diags(np.linspace(1.0, 3.0, 40))
    S = sp.block_diag([L, D]).tocsr()                       # n = 1001 = 62 * 16 + 9
    S.sort_indices()
    A = M.CSR(S.shape[0], S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data.astype(np.float64))
    b = np.random.default_rng(5).uniform(-1, 1, A.n)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x, rep = G.solve(b, method=method, precision=precision, tol=1e-10)
    assert rep["converged"] and rep["relres_true"] <= 1e-10
    assert _relres(A, x, b) <= 1.0001e-10
    if method == "cg" and precision == "fp64":
        T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
        xo, ro = T.cg_fp64(b, tol=1e-10, max_iter=5000)
        np.testing.assert_allclose(x, xo, rtol=0, atol=1e-8 * np.abs(xo).max())
        assert abs(rep["iterations"] - ro["iterations"]) <= 0.05 * ro["iterations"] + 1


@pytest.mark.parametrize("method,precision", [("cg", "fp64"), ("cg", "mixed"), ("bicgstab", "mixed")])
def test_gpu_initial_guess(mf, cuda, p3d, cd3d, method, precision):
    """x0_given: the solve starts from x (r = b - A x in FP64).  From the exact
    solution it stops at once; restarted from a 1e-4 solution it reaches 1e-10
    in fewer iterations than from zero, on host and on device buffers."""
    import torch
    A, b, _ = p3d if method == "cg" else cd3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    xc, rc = G.solve(b, method=method, precision=precision, tol=1e-10)
    assert rc["converged"]
    xs = __import__("scipy.sparse.linalg", fromlist=["spsolve"]).spsolve(A.to_scipy().tocsc(), b)
    x0 = xs.copy()
    x1, r1 = G.solve(b, x0, method=method, precision=precision, tol=1e-10, x0_given=1)
    assert r1["converged"] and r1["iterations"] <= 1 and _relres(A, x1, b) <= 1e-10
    xa, ra = G.solve(b, method=method, precision=precision, tol=1e-4)
    xw, rw = G.solve(b, xa.copy(), method=method, precision=precision, tol=1e-10, x0_given=1)
    assert rw["converged"] and _relres(A, xw, b) <= 1.0001e-10
    assert rw["iterations"] < rc["iterations"], (rw["iterations"], rc["iterations"])
    bd = torch.from_numpy(b).cuda()
    xd = torch.from_numpy(xa).cuda()
    xd, rd = G.solve(bd, xd, method=method, precision=precision, tol=1e-10, x0_given=1)
    assert rd["iterations"] == rw["iterations"]
    np.testing.assert_array_equal(xd.cpu().numpy(), xw)


def test_gpu_relaxed_precision_converges_and_uses_fp16(mf, cuda, p3d):
    """relax_eta: once relax_eta * tol / (||r|| / ||b||) exceeds FP16's unit
    roundoff, the whole SpMV runs on FP16 stored values.  The solve still
    converges on its FP64 true residual (host-checked), FP16 tiles were used,
    and relax_eta = 0 uses none (this system has no exact-FP16 tiles)."""
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x0, r0 = G.solve(b, method="cg", precision="mixed", tol=1e-8)
    assert r0["tile_uses"][2] == 0 and r0["tile_uses"][3] == 0, r0["tile_uses"]
    x, rep = G.solve(b, method="cg", precision="mixed", tol=1e-8, relax_eta=1.0)
    assert rep["converged"] and rep["relres_true"] <= 1e-8
    assert _relres(A, x, b) <= 1.0001e-8
    assert rep["tile_uses"][2] > 0 and rep["tile_uses"][3] == 0, rep["tile_uses"]


def test_gpu_demotion_feedback_turns_unpaid_lookups_off(mf, cuda):
    """Mixed BiCGSTAB on a 48^3 convection-diffusion system: enough of the
    operands' column segments are small that per-slice lookups engage, but a
    slice demotes only when all of its tiles' segments are small, so each
    dynamic SpMV runs few tiles below FP32.  The demotion feedback then turns
    the lookups off for the next 16 SpMVs: the solve runs a small fraction of
    the FP16 / INT8 tile products that the same solve with the gates off
    (demote_min_fraction = 0: every SpMV dynamic) runs.  Both converge on the
    FP64 true residual."""
    from millefeuille import matrices as M
    C, bc, _ = M.convdiff3d(48, seed=2)
    G = mf.Matrix.from_csr(C.n, C.n, C.rowptr, C.colidx, C.val)
    x1, r1 = G.solve(bc, method="bicgstab", precision="mixed", tol=1e-8)
    x0, r0 = G.solve(bc, method="bicgstab", precision="mixed", tol=1e-8, demote_min_fraction=0.0)
    for x, r in ((x1, r1), (x0, r0)):
        assert r["converged"] and _relres(C, x, bc) <= 1.0001e-8, r
    low1 = r1["tile_uses"][2] + r1["tile_uses"][3]
    low0 = r0["tile_uses"][2] + r0["tile_uses"][3]
    assert low0 > 1000 and 0 < low1 < 0.2 * low0, (r1["tile_uses"], r0["tile_uses"])


def test_gpu_fp16_exact_matrix_runs_fp16_lean_walk(mf, cuda):
    """Every tile of the 2D Laplacian (values 4 and -1) is exact in FP16, so the
    mixed mode runs its SpMVs on FP16 stored values through the lookup-free
    walk: no tile product runs in FP32 or FP64, each SpMV counts every tile and
    entry once, and since the values lose nothing the solve takes the FP64
    solve's iterations and agrees with its x.  use_lossless = 0 keeps FP32."""
    from millefeuille import matrices as M
    A, b, _ = M.laplace2d_system(96, seed=0)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    xf, rf = G.solve(b, precision="fp64", tol=1e-10, replace_every=0)
    xm, rm = G.solve(b, precision="mixed", tol=1e-10)
    assert rm["converged"] and _relres(A, xm, b) <= 1.0001e-10, rm
    T = G.info["tilenum"]
    tu, nu = rm["tile_uses"], rm["nnz_uses"]
    assert tu[0] == 0 and tu[1] == 0 and tu[2] > 0, tu
    assert sum(tu) % T == 0 and sum(nu) == sum(tu) // T * A.nnz, (tu, nu)
    assert abs(rm["iterations"] - rf["iterations"]) <= 2, (rm["iterations"], rf["iterations"])
    np.testing.assert_allclose(xm, xf, rtol=0, atol=1e-8 * np.abs(xf).max())
    x2, r2 = G.solve(b, precision="mixed", tol=1e-10, use_lossless=0)
    assert r2["converged"] and r2["tile_uses"][2] == 0 and r2["tile_uses"][1] > 0, r2["tile_uses"]
    # BiCGSTAB takes the same FP16 walk for both of its SpMVs
    x3, r3 = G.solve(b, method="bicgstab", precision="mixed", tol=1e-10)
    assert r3["converged"] and _relres(A, x3, b) <= 1.0001e-10, r3
    assert r3["tile_uses"][0] == 0 and r3["tile_uses"][1] == 0 and r3["tile_uses"][2] > 0, r3["tile_uses"]
