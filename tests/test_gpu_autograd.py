"""Differentiable solve: mf_value_grad, transposed handles and the autograd
wrapper, against dense FP64 linear algebra and central differences.

Tolerances: value gradients from the kernel rtol 1e-14 (one product and a
fixed-order sum per entry); FP64 adjoint gradients 1e-7 of the largest entry
against a dense solve (solver tolerance 1e-12); mixed-precision gradients 1e-5
(solver tolerance 1e-10, FP32 tile products); central differences h = 1e-6,
rel 1e-5 / abs 1e-5 on a 16^2 instance and rel 1e-4 / abs 1e-4 of the
gradient scale on the 64^2 instance (FP64 and mixed solves run to rounding)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.to("cuda:0") if dtype is None else t.to("cuda:0", dtype)


def _rows(A):
    return np.repeat(np.arange(A.n), np.diff(A.rowptr))


def test_value_grad_matches_dense(mf, cuda):
    from millefeuille import matrices as M
    A = M.random_csr(150, 150, 0.05, seed=21, empty_rows=0.1)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    rng = np.random.default_rng(3)
    lam, x = rng.standard_normal((3, A.n)), rng.standard_normal((3, A.n))
    ref = -np.einsum("ke,ke->e", lam[:, _rows(A)], x[:, A.colidx])
    np.testing.assert_allclose(G.value_grad(lam, x), ref, rtol=1e-14, atol=1e-14)
    g1 = G.value_grad(_dev(lam[0]), _dev(x[0])).cpu().numpy()          # device pointers, one rhs
    np.testing.assert_allclose(g1, -lam[0][_rows(A)] * x[0][A.colidx], rtol=1e-14, atol=1e-14)


def test_transposed_handle_matches_scipy(mf, cuda):
    from millefeuille import matrices as M
    A = M.random_csr(120, 90, 0.08, seed=22)
    import scipy.sparse as sp
    S = sp.csr_matrix((A.val, A.colidx, A.rowptr), shape=(120, 90))
    G = mf.Matrix.from_csr(120, 90, A.rowptr, A.colidx, A.val)
    T = G.transposed()
    assert T.info["n_rows"] == 90 and T.info["n_cols"] == 120 and T.info["nnz"] == A.nnz
    y = np.random.default_rng(4).standard_normal(120)
    np.testing.assert_allclose(T.spmv(y), S.T @ y, rtol=1e-13, atol=1e-13 * np.abs(S.T @ y).max())


def _dense_grads(A, b, xt):
    """Dense FP64 reference: x = A^-1 b, L = ||x - xt||^2, lambda = A^-T 2 (x - xt)."""
    D = A.to_scipy().toarray()
    x = np.linalg.solve(D, b)
    lam = np.linalg.solve(D.T, 2.0 * (x - xt))
    return x, lam, -lam[_rows(A)] * x[A.colidx]


@pytest.mark.parametrize("precision,tol,rtol", [("fp64", 1e-12, 1e-7), ("mixed", 1e-10, 1e-5)])
def test_autograd_cg_matches_dense_gradient(mf, cuda, precision, tol, rtol):
    import torch
    from millefeuille import matrices as M
    from millefeuille.autograd import sparse_solve
    A, B, Xt, _ = M.aniso2d_grf(64, seed=4, corr=16.0, nrhs=1)      # the 64^2 check instance: n = 4096
    b, xt = B[0], Xt[0]
    val = _dev(A.val).requires_grad_(True)
    bt = _dev(b).requires_grad_(True)
    x = sparse_solve(_dev(A.rowptr), _dev(A.colidx), val, bt, method="cg", precision=precision, tol=tol)
    loss = ((x - _dev(xt)) ** 2).sum()
    loss.backward()
    x_ref, lam_ref, gval_ref = _dense_grads(A, b, xt)
    np.testing.assert_allclose(x.detach().cpu().numpy(), x_ref, rtol=0, atol=rtol * np.abs(x_ref).max())
    np.testing.assert_allclose(bt.grad.cpu().numpy(), lam_ref, rtol=0, atol=rtol * np.abs(lam_ref).max())
    np.testing.assert_allclose(val.grad.cpu().numpy(), gval_ref, rtol=0, atol=rtol * np.abs(gval_ref).max())


@pytest.mark.parametrize("precision,tol,rtol", [("fp64", 1e-12, 1e-7), ("mixed", 1e-10, 1e-5)])
def test_autograd_cg_many_rhs_batch_matches_dense_gradient(mf, cuda, precision, tol, rtol):
    """More than 8 right-hand sides go through the pattern's tuned one-system
    batch, forward and adjoint (the symmetric adjoint reuses the forward's
    batch); gradients against the dense FP64 ones, summed over the columns."""
    import torch
    from millefeuille import matrices as M
    from millefeuille.autograd import SolvePattern, sparse_solve
    A, B, Xt, _ = M.aniso2d_grf(32, seed=4, corr=8.0, nrhs=12)
    rp, ci = _dev(A.rowptr), _dev(A.colidx)
    pat = SolvePattern(rp, ci, A.n, symmetric=True)
    val = _dev(A.val).requires_grad_(True)
    bt = _dev(B).requires_grad_(True)
    x = sparse_solve(rp, ci, val, bt, method="cg", precision=precision, tol=tol, pattern=pat)
    ((x - _dev(Xt)) ** 2).sum().backward()
    assert len(pat.reports) == 24 and all("item_blocks" in r for r in pat.reports)
    assert all(r["converged"] and r["relres_true"] <= tol for r in pat.reports)
    assert len(pat._batches) == 1
    D = A.to_scipy().toarray()
    X = np.linalg.solve(D, B.T).T
    L = np.linalg.solve(D.T, 2.0 * (X - Xt).T).T
    gval = -np.einsum("ke,ke->e", L[:, _rows(A)], X[:, A.colidx])
    np.testing.assert_allclose(x.detach().cpu().numpy(), X, rtol=0, atol=rtol * np.abs(X).max())
    np.testing.assert_allclose(bt.grad.cpu().numpy(), L, rtol=0, atol=rtol * np.abs(L).max())
    np.testing.assert_allclose(val.grad.cpu().numpy(), gval, rtol=0, atol=rtol * np.abs(gval).max())
    # new values tensor (same values): a new handle and batch, configured from the
    # pair tuned above without timing runs; the same kernels give the same bits
    cfg = dict(pat._configs)
    val2 = _dev(A.val).requires_grad_(True)
    bt2 = _dev(B).requires_grad_(True)
    x2 = sparse_solve(rp, ci, val2, bt2, method="cg", precision=precision, tol=tol, pattern=pat)
    ((x2 - _dev(Xt)) ** 2).sum().backward()
    assert pat._configs == cfg and len(cfg) == 1
    assert torch.equal(x2, x) and torch.equal(val2.grad, val.grad) and torch.equal(bt2.grad, bt.grad)
    pat.close_batches()


def test_autograd_cg_central_differences(mf, cuda):
    import torch
    from millefeuille import matrices as M
    from millefeuille.autograd import SolvePattern, sparse_solve
    A, B, Xt, _ = M.aniso2d_grf(16, seed=4, corr=3.0, nrhs=2)
    rp, ci = _dev(A.rowptr), _dev(A.colidx)
    pat = SolvePattern(rp, ci, A.n, symmetric=True)
    Bt, Xtt = _dev(B), _dev(Xt)

    # a fixed, generous iteration count (n = 256, cond ~ 1e3) makes every solve
    # converged to rounding and a smooth function of the data, so the
    # differences measure the derivative, not the stopping test
    def loss_of(v, bb):
        x = sparse_solve(rp, ci, v, bb, method="cg", precision="fp64", tol=1e-14, pattern=pat,
                         fixed_iters=1, max_iter=400, replace_every=25)
        return ((x - Xtt) ** 2).sum()

    val = _dev(A.val).requires_grad_(True)
    bt = Bt.clone().requires_grad_(True)
    loss_of(val, bt).backward()
    h = 1e-6
    rng = np.random.default_rng(9)
    for e in rng.choice(A.nnz, 6, replace=False):
        vp, vm = _dev(A.val), _dev(A.val)
        vp[e] += h
        vm[e] -= h
        fd = (loss_of(vp, Bt).item() - loss_of(vm, Bt).item()) / (2 * h)
        assert val.grad[e].item() == pytest.approx(fd, rel=1e-5, abs=1e-5)
    for k, i in [(0, 5), (1, 100), (1, 255)]:
        bp, bm = Bt.clone(), Bt.clone()
        bp[k, i] += h
        bm[k, i] -= h
        fd = (loss_of(_dev(A.val), bp).item() - loss_of(_dev(A.val), bm).item()) / (2 * h)
        assert bt.grad[k, i].item() == pytest.approx(fd, rel=1e-5, abs=1e-5)


def test_autograd_bicgstab_uses_transposed_adjoint(mf, cuda):
    import torch
    from millefeuille import matrices as M
    from millefeuille.autograd import sparse_solve
    A, b, _ = M.convdiff3d(10, seed=2)                              # nonsymmetric, n = 1000
    xt = np.random.default_rng(5).standard_normal(A.n)
    val = _dev(A.val).requires_grad_(True)
    bt = _dev(b).requires_grad_(True)
    x = sparse_solve(_dev(A.rowptr), _dev(A.colidx), val, bt, method="bicgstab", precision="fp64", tol=1e-12)
    ((x - _dev(xt)) ** 2).sum().backward()
    x_ref, lam_ref, gval_ref = _dense_grads(A, b, xt)
    np.testing.assert_allclose(bt.grad.cpu().numpy(), lam_ref, rtol=0, atol=1e-7 * np.abs(lam_ref).max())
    np.testing.assert_allclose(val.grad.cpu().numpy(), gval_ref, rtol=0, atol=1e-7 * np.abs(gval_ref).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autograd_cg_central_differences_64(mf, cuda, precision):
    """The 64^2 gradient-check instance (correlation length 16 cells as in the
    512^2 workload): dL/dval and dL/db from the adjoint against central
    differences (h = 1e-6) of solves run for a fixed 3,000 iterations with FP64
    residual replacement every 25, so every solve has converged to rounding
    (a smooth function of the data) in FP64 and in mixed precision alike."""
    from millefeuille import matrices as M
    from millefeuille.autograd import SolvePattern, sparse_solve
    A, B, Xt, _ = M.aniso2d_grf(64, seed=4, corr=16.0, nrhs=2)
    rp, ci = _dev(A.rowptr), _dev(A.colidx)
    pat = SolvePattern(rp, ci, A.n, symmetric=True)
    Bt, Xtt = _dev(B), _dev(Xt)

    def loss_of(v, bb):
        x = sparse_solve(rp, ci, v, bb, method="cg", precision=precision, tol=1e-14, pattern=pat,
                         fixed_iters=1, max_iter=3000, replace_every=25)
        return ((x - Xtt) ** 2).sum()

    val = _dev(A.val).requires_grad_(True)
    bt = Bt.clone().requires_grad_(True)
    loss_of(val, bt).backward()
    gscale_v = float(val.grad.abs().max())
    gscale_b = float(bt.grad.abs().max())
    h = 1e-6
    rng = np.random.default_rng(19)
    for e in rng.choice(A.nnz, 5, replace=False):
        vp, vm = _dev(A.val), _dev(A.val)
        vp[e] += h
        vm[e] -= h
        fd = (loss_of(vp, Bt).item() - loss_of(vm, Bt).item()) / (2 * h)
        assert val.grad[e].item() == pytest.approx(fd, rel=1e-4, abs=1e-4 * gscale_v), (e, fd)
    for k, i in [(0, 17), (1, 2048), (1, 4095)]:
        bp, bm = Bt.clone(), Bt.clone()
        bp[k, i] += h
        bm[k, i] -= h
        fd = (loss_of(_dev(A.val), bp).item() - loss_of(_dev(A.val), bm).item()) / (2 * h)
        assert bt.grad[k, i].item() == pytest.approx(fd, rel=1e-4, abs=1e-4 * gscale_b), (k, i, fd)
