"""Differentiable sparse solve over the C ABI: x = A^-1 b with gradients for b
and for A's stored values.

    x = sparse_solve(rowptr, colidx, val, b, method="cg", precision="mixed")
    loss(x).backward()        # fills val.grad and b.grad

Forward: the single-kernel solve on device pointers -- for CG, mf_solve_multi
(up to 8 right-hand sides in one launch) or, with more than 8, a one-system
mf_batch per tiled handle, tuned once per pattern and right-hand-side count
(work items of up to 8 columns solved concurrently by teams of blocks); one mf_solve per
column for BiCGSTAB.  Backward: the adjoint solve lambda = A^-T dL/dx with the same
kernel -- on A itself for CG (A symmetric), on a transposed handle
(mf_matrix_create_transposed) for BiCGSTAB -- then dL/db = lambda and
dL/dval[e] = -sum_k lambda_k[i] x_k[j] over A's stored pattern (mf_value_grad,
a hand-written kernel).  No counterpart in the reference.

rowptr / colidx are CUDA int32 tensors, val a CUDA float64 tensor of the
stored values (in CSR order), b a CUDA float64 tensor of shape (n,) or
(nrhs, n).  The tiled handle is rebuilt when val changes (its tensor version
counter) and reused otherwise.
"""
from __future__ import annotations

import torch

from . import Batch, Matrix, default_options


class SolvePattern:
    """A sparsity pattern plus the tiled handles built for its current values."""

    def __init__(self, rowptr, colidx, n_rows, n_cols=None, symmetric=True):
        self.rowptr = rowptr
        self.colidx = colidx
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols if n_cols is not None else n_rows)
        self.symmetric = bool(symmetric)
        self._key = None
        self._A = None
        self._AT = None
        self._batches = {}          # (handle, nrhs, precision) -> one-system Batch of the current values
        self._configs = {}          # (rows, cols, nrhs, precision) -> (columns per item, blocks per SM)
        self.reports = []           # per-solve reports of the last forward / backward

    def matrix(self, val) -> Matrix:
        key = (val.data_ptr(), val._version, tuple(val.shape))
        if self._A is None or key != self._key:
            self.close_batches()
            self._A = Matrix.from_csr(self.n_rows, self.n_cols, self.rowptr, self.colidx, val.detach().contiguous())
            self._AT = None
            self._key = key
        return self._A

    def adjoint(self) -> Matrix:
        if self.symmetric:
            return self._A
        if self._AT is None:
            self._AT = self._A.transposed()
        return self._AT

    def batch(self, A: Matrix, nrhs: int, precision: int, stream) -> Batch:
        """The one-system batch of A with nrhs right-hand sides, kept until the
        values change.  The first batch of a column count and precision is
        tuned (mf_batch_tune: columns per work item, blocks per SM); later ones
        (new values, same pattern and sizes) take the same pair
        (mf_batch_configure) without timing runs."""
        key = (id(A), int(nrhs), int(precision))
        bt = self._batches.get(key)
        if bt is None:
            bt = Batch([A], [int(nrhs)], stream=stream)
            ckey = (A.info["n_rows"], A.info["n_cols"], key[1], key[2])
            if ckey in self._configs:
                bt.configure(*self._configs[ckey], stream=stream)
            else:
                bt.tune(key[2], stream=stream)
                self._configs[ckey] = bt.config()
            self._batches[key] = bt
        return bt

    def close_batches(self) -> None:
        for bt in self._batches.values():
            bt.close()
        self._batches = {}


# More right-hand sides than one multi-column launch takes: a one-system batch.
# Its work items (up to 8 columns each) run concurrently on teams of blocks,
# where mf_solve_multi would run one 8-column group after another on the
# whole grid (32 columns of the 512^2 anisotropic system: 1.62 s against 2.0 s).
_BATCH_ABOVE = 8


def _solve_all(A: Matrix, B, opts, reports, pattern: "SolvePattern"):
    """All right-hand sides: for CG in the FP64 / mixed modes, mf_solve_multi
    (up to 8) or the pattern's tuned one-system batch (more than 8); one
    mf_solve per column otherwise."""
    X = torch.zeros_like(B)
    if B.shape[0] > 1 and opts.method == 0 and opts.precision in (0, 1):
        if B.shape[0] > _BATCH_ABOVE:
            stream = torch.cuda.current_stream(B.device).cuda_stream
            bt = pattern.batch(A, B.shape[0], opts.precision, stream)
            _, reps = bt.solve([B], [X], options=opts, use_graph=False, stream=stream)
            reports.extend(reps[0])
            return X
        _, reps = A.solve_multi(B, X, options=opts)
        reports.extend(reps)
        return X
    for k in range(B.shape[0]):
        _, rep = A.solve(B[k], X[k], options=opts)
        reports.append(rep)
    return X


class _SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, val, b, pattern: SolvePattern, opts):
        A = pattern.matrix(val)
        B = b.detach().reshape(-1, b.shape[-1]).contiguous()
        pattern.reports = []
        X = _solve_all(A, B, opts, pattern.reports, pattern)
        ctx.pattern, ctx.opts = pattern, opts
        ctx.save_for_backward(X)
        ctx.bshape = b.shape
        return X.reshape(b.shape)

    @staticmethod
    def backward(ctx, gx):
        (X,) = ctx.saved_tensors
        pattern, opts = ctx.pattern, ctx.opts
        G = gx.detach().reshape(X.shape).contiguous()
        AT = pattern.adjoint()
        lam = _solve_all(AT, G, opts, pattern.reports, pattern)
        grad_val = grad_b = None
        if ctx.needs_input_grad[0]:
            grad_val = pattern._A.value_grad(lam, X)
        if ctx.needs_input_grad[1]:
            grad_b = lam.reshape(ctx.bshape)
        return grad_val, grad_b, None, None


def sparse_solve(rowptr, colidx, val, b, *, n_cols=None, method="cg", precision="mixed", tol=1e-8,
                 symmetric=None, pattern: SolvePattern | None = None, **options):
    """x = A^-1 b, differentiable in val and b (see the module docstring).

    symmetric defaults to True for CG and False for BiCGSTAB; pass a
    SolvePattern to reuse handles (and read .reports) across calls."""
    if symmetric is None:
        symmetric = (method == "cg")
    if pattern is None:
        pattern = SolvePattern(rowptr, colidx, rowptr.numel() - 1, n_cols, symmetric)
    opts = default_options(method=method, precision=precision, tol=tol, **options)
    return _SparseSolve.apply(val, b, pattern, opts)
