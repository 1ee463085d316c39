"""mf_spmv_noalloc: the allocation-free y = A x entry point, checked against
mf_spmv (the existing entry point) on the same inputs.

Collected last on purpose (file name): it must pass on its own and after every
other GPU test has used the library.  Tolerance: FP64 rtol 1e-13 and FP32
tiles rtol 1e-6 of max|y| -- both calls run the same slice kernel on the same
padded operand, so the results agree to rounding of identical arithmetic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def _check(y, y_ref, precision):
    tol = 1e-13 if precision == "fp64" else 1e-6
    np.testing.assert_allclose(y, y_ref, rtol=tol, atol=tol * np.abs(y_ref).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_spmv_matches_spmv_two_calls_in_a_row(mf, cuda, precision):
    import torch
    from millefeuille import matrices as M
    # rectangular, column count not a multiple of 16, unsorted columns, empty rows:
    # the padded operand tail is exercised
    A = M.random_csr(200, 230, 0.05, seed=11, empty_rows=0.1)
    B, _, _ = M.poisson3d_varcoef(24, seed=1)          # a larger system first, so the
    GA = mf.Matrix.from_csr(A.n, 230, A.rowptr, A.colidx, A.val)   # scratch holds stale data
    GB = mf.Matrix.from_csr(B.n, B.n, B.rowptr, B.colidx, B.val)
    rng = np.random.default_rng(5)
    xb = _dev(rng.uniform(-1, 1, B.n))
    x1 = _dev(rng.uniform(-1, 1, 230))
    x2 = _dev(rng.uniform(-1, 1, 230))
    # references through the existing entry point
    yb_ref = GB.spmv(xb, precision=precision).cpu().numpy()
    y1_ref = GA.spmv(x1, precision=precision).cpu().numpy()
    y2_ref = GA.spmv(x2, precision=precision).cpu().numpy()
    yb = torch.empty(B.n, dtype=torch.float64, device="cuda:0")
    y1 = torch.empty(A.n, dtype=torch.float64, device="cuda:0")
    y2 = torch.empty(A.n, dtype=torch.float64, device="cuda:0")
    s = torch.cuda.current_stream().cuda_stream
    GB.spmv_noalloc(xb, yb, precision=precision, stream=s)
    GA.spmv_noalloc(x1, y1, precision=precision, stream=s)    # two calls in a row on one stream
    GA.spmv_noalloc(x2, y2, precision=precision, stream=s)
    torch.cuda.synchronize()
    _check(yb.cpu().numpy(), yb_ref, precision)
    _check(y1.cpu().numpy(), y1_ref, precision)
    _check(y2.cpu().numpy(), y2_ref, precision)
    # and against the FP64 CSR product
    if precision == "fp64":
        import scipy.sparse as sp
        S = sp.csr_matrix((A.val, A.colidx, A.rowptr), shape=(A.n, 230))
        _check(y1.cpu().numpy(), S @ x1.cpu().numpy(), precision)


def test_noalloc_spmv_leaves_free_device_memory_unchanged(mf, cuda):
    import torch
    from millefeuille import matrices as M
    B, _, _ = M.poisson3d_varcoef(20, seed=1)
    G = mf.Matrix.from_csr(B.n, B.n, B.rowptr, B.colidx, B.val)
    x = _dev(np.random.default_rng(6).uniform(-1, 1, B.n))
    y = torch.empty(B.n, dtype=torch.float64, device="cuda:0")
    G.spmv_noalloc(x, y)                   # first call on the device: one-time scratch lookup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for prec in ("fp64", "mixed", "fp64"):
        G.spmv_noalloc(x, y, precision=prec)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    np.testing.assert_allclose(y.cpu().numpy(), B.matvec(x.cpu().numpy()), rtol=1e-13,
                               atol=1e-13 * np.abs(y.cpu().numpy()).max())


def test_noalloc_spmv_rejects_oversize_matrix(mf, cuda):
    import torch
    n = (1 << 21) + 16                 # one tile-row past MF_SPMV_NOALLOC_MAX_LEN
    rowptr = np.arange(n + 1, dtype=np.int32)
    colidx = np.arange(n, dtype=np.int32)
    G = mf.Matrix.from_csr(n, n, rowptr, colidx, np.full(n, 2.0))
    x = torch.ones(n, dtype=torch.float64, device="cuda:0")
    y = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    with pytest.raises(mf.MFError) as e:
        G.spmv_noalloc(x, y)
    assert e.value.status == 5          # MF_ERR_UNSUPPORTED, nothing launched
    assert float(y.abs().max()) == 0.0
