"""The smallest systems the solvers take: one row, a single partial tile-row,
exactly one full tile-row, one row past it, a few tile-rows.  Every method and
precision converges on its FP64 true residual and agrees with a dense FP64
solve; the FP64 and FP32 SpMVs agree with the dense product.  Most of the
persistent grid's half-warps own no tile-row here, and the operand's last
segment is mostly padding.

Tolerances: solves to relres 1e-12 (FP64) and 1e-10 (mixed), checked with an
independent FP64 residual; x within 1e-8 of the dense solution relative to its
largest entry (these systems have condition numbers below 10); SpMV FP64
rtol 1e-13, FP32 values rtol 1e-6 against the product of the FP32-rounded
matrix."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = (1, 2, 7, 16, 17, 40)


def _system(n, symmetric, seed):
    """Diagonally dominant with couplings inside and across tile-rows (row i
    to i +- 1 and i +- 16 where they exist); unsymmetric couplings for BiCGSTAB."""
    from millefeuille import matrices as M
    rng = np.random.default_rng(seed)
    D = np.zeros((n, n))
    for i in range(n):
        for j in (i - 16, i - 1, i + 1, i + 16):
            if 0 <= j < n and (symmetric is False or j > i):
                D[i, j] = -rng.uniform(0.2, 1.0)
    if symmetric:
        D = D + D.T
    D[np.arange(n), np.arange(n)] = np.abs(D).sum(axis=1) + rng.uniform(0.5, 2.0, n)
    rp, ci, va = [0], [], []
    for i in range(n):
        nz = np.nonzero(D[i])[0]
        ci.extend(nz.tolist())
        va.extend(D[i, nz].tolist())
        rp.append(len(ci))
    A = M.CSR(n, np.asarray(rp, dtype=np.int32), np.asarray(ci, dtype=np.int32), np.asarray(va))
    b = rng.uniform(-1, 1, n)
    return A, D, b


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("method,precision", [("cg", "fp64"), ("cg", "mixed"), ("bicgstab", "fp64"),
                                              ("bicgstab", "mixed")])
def test_small_system_solves(mf, cuda, n, method, precision):
    A, D, b = _system(n, method == "cg", seed=100 + n)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    tol = 1e-12 if precision == "fp64" else 1e-10
    x, rep = G.solve(b, method=method, precision=precision, tol=tol)
    xd = np.linalg.solve(D, b)
    assert rep["converged"] and rep["relres_true"] <= tol
    assert np.linalg.norm(D @ x - b) <= 1.0001 * tol * np.linalg.norm(b)
    np.testing.assert_allclose(x, xd, rtol=0, atol=1e-8 * np.abs(xd).max())


@pytest.mark.parametrize("n", SIZES)
def test_small_system_spmv(mf, cuda, n):
    A, D, _ = _system(n, False, seed=200 + n)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    x = np.random.default_rng(n).standard_normal(n)
    y_ref = D @ x
    np.testing.assert_allclose(G.spmv(x, precision="fp64"), y_ref, rtol=1e-13, atol=1e-13 * np.abs(y_ref).max())
    y32_ref = D.astype(np.float32).astype(np.float64) @ x
    np.testing.assert_allclose(G.spmv(x, precision="mixed"), y32_ref, rtol=1e-6, atol=1e-6 * np.abs(y_ref).max())
