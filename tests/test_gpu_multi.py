"""CG on several right-hand sides in one persistent launch (mf_solve_multi)
against the single-column kernel and the FP64 oracle.

Tolerances: every column converges to its own relres target on the FP64 true
residual; columns agree with single-column solves to 1e-7 of max|x| at
tol 1e-10 (same algorithm, different reduction grid, so the last bits and the
iteration count may differ: iterations within 5 % + 2)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def p3d():
    from millefeuille import matrices as M
    return M.poisson3d_varcoef(24, seed=1)


def _relres(A, x, b):
    return np.linalg.norm(A.to_scipy() @ x - b) / np.linalg.norm(b)


@pytest.mark.parametrize("nrhs", [2, 3, 8, 11])
def test_multi_fp64_matches_single_column_solves(mf, cuda, p3d, nrhs):
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    rng = np.random.default_rng(nrhs)
    B = rng.standard_normal((nrhs, A.n))
    B[0] = b
    X, reps = G.solve_multi(B, method="cg", precision="fp64", tol=1e-10)
    assert len(reps) == nrhs
    for k in range(nrhs):
        xs, rs = G.solve(B[k], method="cg", precision="fp64", tol=1e-10)
        assert reps[k]["converged"] and reps[k]["relres_true"] <= 1e-10
        assert _relres(A, X[k], B[k]) <= 1.0001e-10
        assert abs(reps[k]["iterations"] - rs["iterations"]) <= 2 + 0.05 * rs["iterations"]
        np.testing.assert_allclose(X[k], xs, rtol=0, atol=1e-7 * np.abs(xs).max())


def test_multi_mixed_converges_and_zero_column(mf, cuda, p3d):
    import torch
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    B = np.random.default_rng(7).standard_normal((5, A.n))
    B[3] = 0.0                                   # a zero column: x = 0, converged at once
    Bd = torch.from_numpy(B).cuda()
    X, reps = G.solve_multi(Bd, method="cg", precision="mixed", tol=1e-8)
    X = X.cpu().numpy()
    for k in range(5):
        assert reps[k]["converged"]
        if k == 3:
            assert reps[k]["iterations"] == 0 and not np.any(X[k])
        else:
            assert reps[k]["relres_true"] <= 1e-8 and _relres(A, X[k], B[k]) <= 1.0001e-8


def test_multi_is_deterministic(mf, cuda, p3d):
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    B = np.random.default_rng(8).standard_normal((4, A.n))
    X1, r1 = G.solve_multi(B, method="cg", precision="mixed", tol=1e-8)
    X2, r2 = G.solve_multi(B, method="cg", precision="mixed", tol=1e-8)
    assert [r["iterations"] for r in r1] == [r["iterations"] for r in r2]
    np.testing.assert_array_equal(X1, X2)


def test_multi_rejects_parity_and_bicgstab(mf, cuda, p3d):
    A, b, _ = p3d
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    B = np.random.default_rng(9).standard_normal((2, A.n))
    for kw in ({"method": "bicgstab"}, {"method": "cg", "precision": "parity"}):
        with pytest.raises(mf.MFError) as e:
            G.solve_multi(B, **kw)
        assert e.value.status == 5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_multi_initial_guess(mf, cuda, p3d, precision):
    """x0_given for several right-hand sides: X starts from the given columns
    (R = B - A X in FP64).  Warm-started from 1e-4 solutions the columns reach
    1e-10 in fewer iterations than from zero; the exact solutions stop at once;
    host and device buffers give the same bits."""
    import torch
    import scipy.sparse.linalg as sla
    A, b, _ = p3d
    rng = np.random.default_rng(9)
    B = np.stack([b, rng.standard_normal(A.n), rng.standard_normal(A.n)])
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    Xc, rc = G.solve_multi(B, method="cg", precision=precision, tol=1e-10)
    Xa, _ = G.solve_multi(B, method="cg", precision=precision, tol=1e-4)
    Xw, rw = G.solve_multi(B, Xa.copy(), method="cg", precision=precision, tol=1e-10, x0_given=1)
    S = A.to_scipy()
    for k in range(3):
        assert rw[k]["converged"] and np.linalg.norm(S @ Xw[k] - B[k]) / np.linalg.norm(B[k]) <= 1.0001e-10
        assert rw[k]["iterations"] < rc[k]["iterations"], (k, rw[k]["iterations"], rc[k]["iterations"])
    Xs = np.stack([sla.spsolve(S.tocsc(), B[k]) for k in range(3)])
    _, re = G.solve_multi(B, Xs.copy(), method="cg", precision=precision, tol=1e-10, x0_given=1)
    assert all(r["converged"] and r["iterations"] <= 1 for r in re)
    Xd, rd = G.solve_multi(torch.from_numpy(B).cuda(), torch.from_numpy(Xa).cuda(), method="cg",
                           precision=precision, tol=1e-10, x0_given=1)
    assert [r["iterations"] for r in rd] == [r["iterations"] for r in rw]
    np.testing.assert_array_equal(Xd.cpu().numpy(), Xw)
