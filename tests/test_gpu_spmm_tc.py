"""The tensor-core experiment for 8 right-hand sides (mf_debug_spmm): the
CUDA-core product of FP16 stored values against FP64 X, and the tensor-core
product (tiles densified in shared memory, X rounded to FP16, FP32
accumulation by mma.sync.m16n8k16), both against the FP64 product of the
FP16-rounded values.  Tolerances, relative to sum |a| |x| per row: CUDA cores
1e-14 (FP64 sums of the same products); tensor cores 2^-10 (X rounded to FP16,
2^-11, plus FP32 accumulation)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _f16_values(A):
    return A.val.astype(np.float32).astype(np.float16).astype(np.float64)


@pytest.mark.parametrize("case", ["aniso2d_64", "random_wide"])
def test_spmm8_cuda_and_tensor_cores_match_fp64(mf, cuda, case):
    import scipy.sparse as sp
    from millefeuille import matrices as M
    if case == "aniso2d_64":
        A = M.aniso2d_grf(64, seed=4, corr=16.0, nrhs=1)[0]
        ncols = A.n
    else:                                        # rows over several slices, ragged last tile-row
        A = M.random_csr(500, 530, 0.06, seed=4)
        ncols = 530
    G = mf.Matrix.from_csr(A.n, ncols, A.rowptr, A.colidx, A.val)
    X = np.random.default_rng(3).uniform(-1, 1, (8, ncols))
    S16 = sp.csr_matrix((_f16_values(A), A.colidx, A.rowptr), shape=(A.n, ncols))
    Yref = (S16 @ X.T).T
    scale = (abs(S16) @ np.abs(X).T).T
    Ycc, _ = G.spmm8(X, tensor_cores=False)
    assert np.all(np.abs(Ycc - Yref) <= 1e-14 * scale + 1e-300)
    Ytc, _ = G.spmm8(X, tensor_cores=True)
    assert np.all(np.abs(Ytc - Yref) <= 2.0 ** -10 * scale + 1e-300)
    assert np.abs(Ytc - Yref).max() > 0          # the tensor-core path did round X to FP16
