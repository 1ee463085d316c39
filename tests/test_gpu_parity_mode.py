"""Parity of the reduced-precision tile products and of the parity-mode solver.

1. Every stored precision of the tile SpMV against the oracle's product of the
   same encoded values (orc_spmv_slices): FP64, FP32 (Val_Low), FP16 (the
   reference encoder's half, RN of the float) and scaled INT8, each widened to
   FP64 against the FP64 x and summed in the slice walk's entry order.  The
   GPU and the oracle run the same fma sequence, so y must match bit for bit.

2. The parity-mode CG (MF_PREC_PARITY: the reference's label rule and tile
   arithmetic of main-cg-mixed.cu:1115-1385 -- FP32 fmaf, FP16 __hfma on
   half(p), INT8 int8 sums of truncated values, bypass skipped, even / odd
   partials per (tile, row), labels from |p_new - p_old|) against the oracle's
   restatement orc_cg_parity, after k = 1, 5 and 20 fixed iterations on
   systems whose right-hand side is scaled so that the labels spread over
   FP64 / FP32 / FP16 / INT8 / bypass.  The labels the GPU leaves for the next
   SpMV must equal the oracle's segment for segment; x agrees to a stated
   tolerance (the dot products are summed in different orders, so x differs by
   rounding that the FP16 / INT8 arithmetic can amplify)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems():
    from millefeuille import matrices as M
    A1, _, _ = M.poisson3d_varcoef(12, seed=1)
    A2 = M.laplace2d(24)
    # wide rows: more than 15 tiles per tile-row, so rows span several slices;
    # 530 columns and 500 rows leave a ragged last tile-row
    A3 = M.random_csr(500, 530, 0.06, seed=4)
    return [("poisson3d_12", A1, A1.n), ("laplace2d_24", A2, A2.n), ("random_500x530", A3, 530)]


@pytest.mark.parametrize("prec", [0, 1, 2, 3])
def test_gpu_spmv_tiles_bit_exact_vs_oracle(mf, oracle_mod, cuda, prec):
    import scipy.sparse as sp
    for name, A, ncols in _systems():
        G = mf.Matrix.from_csr(A.n, ncols, A.rowptr, A.colidx, A.val)
        T = oracle_mod.Tiles(A.n, ncols, A.rowptr, A.colidx, A.val)
        x = np.random.default_rng(11).uniform(-1, 1, ncols)
        y = G.spmv_tiles(x, prec)
        yo = T.spmv_slices(x, prec)
        np.testing.assert_array_equal(y, yo, err_msg=f"{name} tile precision {prec}")
        # and, for the floating-point encodings, close to the exact product within
        # the stored precision's rounding (unit roundoff x sum |a| |x|, plus the
        # FP64 sum's own rounding)
        if prec < 3:
            S = sp.csr_matrix((A.val, A.colidx, A.rowptr), shape=(A.n, ncols))
            ye = S @ x
            scale = abs(S) @ np.abs(x)
            rel = {0: 1e-14, 1: 1.2e-7, 2: 1e-3}[prec]
            assert np.all(np.abs(y - ye) <= rel * scale), (name, prec)


def _parity_cases():
    from millefeuille import matrices as M
    A1, b1, _ = M.poisson3d_varcoef(12, seed=1)
    A2, b2, _ = M.laplace2d_system(24, seed=0)
    return [("poisson3d_12 b x 1e-6", A1, b1 * 1e-6), ("poisson3d_12 b x 3e-6", A1, b1 * 3e-6),
            ("laplace2d_24 b x 2e-6", A2, b2 * 2e-6)]


def test_gpu_parity_cg_labels_and_x_match_oracle(mf, oracle_mod, cuda):
    seen = set()
    for name, A, b in _parity_cases():
        G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
        T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
        for k in (1, 5, 20):
            x, rep = G.solve(b, method="cg", precision="parity", max_iter=k, fixed_iters=1, replace_every=0)
            lab = G.solver_labels()
            xo, lab_o, agree, ro = T.cg_parity(b, k)
            assert rep["iterations"] == k
            seen.update(lab_o.tolist())
            mism = np.flatnonzero(lab != lab_o)
            assert mism.size == 0, (name, k, mism[:10], lab[mism[:10]], lab_o[mism[:10]])
            # every lane agreeing: the reference's own (racy) rule is determined there
            np.testing.assert_array_equal(lab[agree], lab_o[agree])
            err = np.linalg.norm(x - xo) / np.linalg.norm(xo)
            assert err <= (1e-12 if k == 1 else 1e-9 if k == 5 else 1e-6), (name, k, err)
    # the cases reach every label class: FP64, FP32, FP16, INT8
    assert {0, 2, 3, 4} <= seen, seen
