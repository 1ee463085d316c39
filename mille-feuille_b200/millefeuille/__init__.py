"""millefeuille -- B200 (sm_100a) tile-grained mixed-precision single-kernel
CG / BiCGSTAB, a drop-in for Mille-feuille's solver path.

Host-side mirror of the C ABI (include/millefeuille.h):

    A = Matrix.from_csr(n_rows, n_cols, rowptr, colidx, val)   # GPU csr2block + encoder
    x, rep = A.solve(b, method="cg", precision="mixed", tol=1e-8)
    y = A.spmv(x)
    A.export("tile_ptr")                                     # reference-layout arrays

Inputs may be numpy arrays (host) or CUDA torch tensors (device, float64 /
int32).  All compute runs in libmillefeuille.so; nothing here falls back to
the CPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (MF_METHOD_BICGSTAB, MF_METHOD_CG, MF_PREC_FP64, MF_PREC_MIXED, MF_PREC_PARITY, MFError,
                   Options, Report, check)

__all__ = ["Matrix", "Batch", "Options", "Report", "MFError", "default_options", "read_matrix", "write_cbd",
           "MF_PREC_FP64", "MF_PREC_MIXED", "MF_PREC_PARITY", "MF_METHOD_CG", "MF_METHOD_BICGSTAB"]

_PREC = {"fp64": MF_PREC_FP64, "mixed": MF_PREC_MIXED, "parity": MF_PREC_PARITY}
_METHOD = {"cg": MF_METHOD_CG, "bicgstab": MF_METHOD_BICGSTAB}

# dtype of every reference-layout array mf_tile_export can return
EXPORT_DTYPES = {
    "tile_ptr": np.int32, "tile_columnidx": np.int32, "tile_nnz": np.int32, "blknnz": np.int32,
    "csr_offset": np.int32, "csrptr_offset": np.int32, "ptroffset1": np.int32, "ptroffset2": np.int32,
    "val": np.float64, "val_low": np.float32, "col": np.uint8, "ptr": np.uint8,
    "nonzero_row_new": np.int32, "blockrowid_new": np.uint8, "blockcsr_ptr_new": np.uint8,
    "tile_rowidx": np.int32, "block_signal": np.int32, "blkcoostylerowidx": np.uint32,
    "colstart": np.int32, "colstop": np.int32, "val_f16": np.uint16, "val_i8_ref": np.int8,
    "val_i8": np.int8, "i8_scale": np.float32, "tile_caps": np.uint8, "seg_ptr": np.int32,
    "seg_kp": np.int32, "seg_rowlen": np.uint16, "seg_off": np.int64, "meta": np.uint8, "v64": np.float64,
    "v32": np.float32, "seg_hdr": np.int32,
}


def default_options(**kw) -> Options:
    o = Options()
    _lib.load().mf_options_default(C.byref(o))
    for k, v in kw.items():
        if k == "precision" and isinstance(v, str):
            v = _PREC[v]
        if k == "method" and isinstance(v, str):
            v = _METHOD[v]
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def _is_cuda_tensor(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _ptr(a):
    if a is None:
        return None
    if _is_cuda_tensor(a):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


class Matrix:
    """Device-resident tiled matrix (an mf_matrix handle)."""

    def __init__(self, handle, keep=None):
        self._h = handle
        self._keep = keep

    @classmethod
    def from_csr(cls, n_rows, n_cols, rowptr, colidx, val, val_low=None, stream=None) -> "Matrix":
        L = _lib.load()
        dev = _is_cuda_tensor(rowptr)
        if not dev:
            rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
            colidx = np.ascontiguousarray(colidx, dtype=np.int32)
            val = np.ascontiguousarray(val, dtype=np.float64)
            if val_low is not None:
                val_low = np.ascontiguousarray(val_low, dtype=np.float32)
        nnz = int(colidx.numel() if dev else colidx.size)
        h = C.c_void_p()
        check(L.mf_matrix_create(C.byref(h), int(n_rows), int(n_cols), nnz, _ptr(rowptr), _ptr(colidx), _ptr(val),
                                 _ptr(val_low), int(dev), C.c_void_p(stream) if stream else None),
              "mf_matrix_create")
        return cls(h)

    def close(self) -> None:
        if self._h:
            _lib.load().mf_matrix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def info(self) -> dict:
        inf = _lib.MatrixInfo()
        check(_lib.load().mf_matrix_get_info(self._h, C.byref(inf)), "mf_matrix_get_info")
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    def export(self, name: str) -> np.ndarray:
        L = _lib.load()
        nb = C.c_size_t()
        check(L.mf_tile_array_bytes(self._h, name.encode(), C.byref(nb)), f"mf_tile_array_bytes({name})")
        dt = np.dtype(EXPORT_DTYPES[name])
        out = np.zeros(nb.value // dt.itemsize, dtype=dt)
        check(L.mf_tile_export(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), nb.value),
              f"mf_tile_export({name})")
        return out

    def solve(self, b, x=None, options: Options | None = None, stream=None, **kw):
        """Solve A x = b.  b: numpy float64 (host) or CUDA float64 tensor
        (device).  Returns (x, report dict); raises MFError on failure
        (the report is attached as err.report)."""
        L = _lib.load()
        o = options if options is not None else default_options(**kw)
        if options is not None and kw:
            for k, v in kw.items():
                setattr(o, k, _PREC.get(v, v) if k == "precision" else _METHOD.get(v, v) if k == "method" else v)
        dev = _is_cuda_tensor(b)
        if x is None:
            if dev:
                import torch
                x = torch.zeros_like(b)
            else:
                b = np.ascontiguousarray(b, dtype=np.float64)
                x = np.zeros_like(b)
        rep = Report()
        st = L.mf_solve(self._h, _ptr(b), _ptr(x), C.byref(o), C.byref(rep), int(dev),
                        C.c_void_p(stream) if stream else None)
        if st != _lib.MF_SUCCESS:
            err = MFError(st, "mf_solve")
            err.report = rep.as_dict()
            raise err
        return x, rep.as_dict()

    def solve_multi(self, B, X=None, options: Options | None = None, stream=None, **kw):
        """Solve A X = B for the rows of B (shape (nrhs, n)) with mf_solve_multi:
        up to 8 right-hand sides per persistent launch.  Returns (X, list of
        report dicts); raises MFError on failure (reports attached)."""
        L = _lib.load()
        o = options if options is not None else default_options(**kw)
        if options is not None and kw:
            for k, v in kw.items():
                setattr(o, k, _PREC.get(v, v) if k == "precision" else _METHOD.get(v, v) if k == "method" else v)
        dev = _is_cuda_tensor(B)
        if dev:
            import torch
            B = B.contiguous()
            if X is None:
                X = torch.zeros_like(B)
        else:
            B = np.ascontiguousarray(B, dtype=np.float64)
            if X is None:
                X = np.zeros_like(B)
        nrhs = int(B.shape[0])
        reps = (Report * nrhs)()
        st = L.mf_solve_multi(self._h, nrhs, _ptr(B), _ptr(X), C.byref(o), reps, int(dev),
                              C.c_void_p(stream) if stream else None)
        out = [r.as_dict() for r in reps]
        if st != _lib.MF_SUCCESS:
            err = MFError(st, "mf_solve_multi")
            err.report = out
            raise err
        return X, out

    def spmv(self, x, y=None, precision="fp64", stream=None):
        L = _lib.load()
        dev = _is_cuda_tensor(x)
        n_rows = self.info["n_rows"]
        if y is None:
            if dev:
                import torch
                y = torch.empty(n_rows, dtype=torch.float64, device=x.device)
            else:
                x = np.ascontiguousarray(x, dtype=np.float64)
                y = np.zeros(n_rows, dtype=np.float64)
        ms = C.c_double()
        check(L.mf_spmv(self._h, _ptr(x), _ptr(y), _PREC[precision] if isinstance(precision, str) else precision,
                        int(dev), C.c_void_p(stream) if stream else None, C.byref(ms)), "mf_spmv")
        self.last_spmv_ms = ms.value
        return y

    def spmv_tiles(self, x, tile_prec):
        """Test hook (mf_debug_spmv_tiles): y = A x with every tile stored in
        one precision -- 0 FP64, 1 FP32, 2 FP16, 3 scaled INT8 -- widened to
        FP64 against the FP64 x.  Host arrays."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.info["n_rows"], dtype=np.float64)
        check(_lib.load().mf_debug_spmv_tiles(self._h, _ptr(x), _ptr(y), int(tile_prec), 0), "mf_debug_spmv_tiles")
        return y

    def spmm8(self, X, tensor_cores=False):
        """Experiment hook (mf_debug_spmm): Y = A X for 8 right-hand sides (rows
        of X, shape (8, n_cols)) with FP16 stored values, on the CUDA cores or
        the tensor cores.  Returns (Y, kernel ms).  Host arrays or CUDA tensors."""
        dev = _is_cuda_tensor(X)
        if dev:
            import torch
            X = X.contiguous()
            Y = torch.empty((8, self.info["n_rows"]), dtype=torch.float64, device=X.device)
        else:
            X = np.ascontiguousarray(X, dtype=np.float64)
            Y = np.zeros((8, self.info["n_rows"]), dtype=np.float64)
        if tuple(X.shape) != (8, self.info["n_cols"]):
            raise ValueError("spmm8 takes X of shape (8, n_cols)")
        ms = C.c_double()
        check(_lib.load().mf_debug_spmm(self._h, _ptr(X), _ptr(Y), int(bool(tensor_cores)), int(dev), C.byref(ms)),
              "mf_debug_spmm")
        return Y, ms.value

    def solver_labels(self):
        """Test hook (mf_debug_solver_labels): the labels the last parity-mode
        solve left for the next SpMV, one per column segment (d_vis codes)."""
        n = self.info["tilen"]
        vis = np.zeros(max(n, 1), dtype=np.int32)
        check(_lib.load().mf_debug_solver_labels(self._h, _ptr(vis), n), "mf_debug_solver_labels")
        return vis[:n]

    def transposed(self, stream=None) -> "Matrix":
        """A handle for A^T (mf_matrix_create_transposed)."""
        L = _lib.load()
        h = C.c_void_p()
        check(L.mf_matrix_create_transposed(C.byref(h), self._h, C.c_void_p(stream) if stream else None),
              "mf_matrix_create_transposed")
        return Matrix(h)

    def value_grad(self, lam, x, out=None, stream=None):
        """dL/dA on the stored pattern: out[e] = -sum_k lam[k, i] x[k, j] for each
        stored entry e = (i, j) (mf_value_grad).  lam: (n_rows,) or (nrhs, n_rows),
        x: (n_cols,) or (nrhs, n_cols); numpy arrays or CUDA tensors (not mixed)."""
        L = _lib.load()
        dev = _is_cuda_tensor(lam)
        nrhs = 1 if lam.ndim == 1 else int(lam.shape[0])
        nnz = int(self.info["nnz"])
        if dev:
            import torch
            lam = lam.contiguous()
            x = x.contiguous()
            if out is None:
                out = torch.empty(nnz, dtype=torch.float64, device=lam.device)
        else:
            lam = np.ascontiguousarray(lam, dtype=np.float64)
            x = np.ascontiguousarray(x, dtype=np.float64)
            if out is None:
                out = np.empty(nnz, dtype=np.float64)
        check(L.mf_value_grad(self._h, nrhs, _ptr(lam), _ptr(x), _ptr(out), int(dev),
                              C.c_void_p(stream) if stream else None), "mf_value_grad")
        return out

    def spmv_noalloc(self, x, y, precision="fp64", stream=None):
        """y = A x through mf_spmv_noalloc: CUDA tensors only, asynchronous on
        `stream`, no allocation inside the call (fixed scratch in the library).

        The kernel writes n_rows doubles into y and the call copies n_cols
        doubles out of x without any bounds of its own, so both tensors are
        checked here before anything is launched: float64, contiguous, at least
        n_cols / n_rows elements, on the device the matrix was built on.  The
        call runs with that device current."""
        import torch
        L = _lib.load()
        if not (_is_cuda_tensor(x) and _is_cuda_tensor(y)):
            raise TypeError("spmv_noalloc takes CUDA tensors for x and y")
        inf = self.info
        for nm, t, need in (("x", x, inf["n_cols"]), ("y", y, inf["n_rows"])):
            if t.dtype != torch.float64:
                raise TypeError(f"spmv_noalloc: {nm} must be float64, got {t.dtype}")
            if not t.is_contiguous():
                raise ValueError(f"spmv_noalloc: {nm} must be contiguous")
            if t.numel() < need:
                raise ValueError(f"spmv_noalloc: {nm} has {t.numel()} elements, needs {need}")
        if x.device != y.device:
            raise ValueError(f"spmv_noalloc: x on {x.device}, y on {y.device}")
        dev = inf["device"]
        if x.device.index != dev:
            raise ValueError(f"spmv_noalloc: tensors on {x.device}, the matrix lives on cuda:{dev}")
        with torch.cuda.device(dev):
            check(L.mf_spmv_noalloc(self._h, _ptr(x), _ptr(y),
                                    _PREC[precision] if isinstance(precision, str) else precision,
                                    C.c_void_p(stream) if stream else None), "mf_spmv_noalloc")
        return y



class Batch:
    """Many independent systems solved in one persistent launch (mf_batch_*).

        batch = Batch([A0, A1, ...], nrhs=[3, 1, ...])      # Matrix handles
        batch.tune("mixed")                                 # right-hand sides per work item
        Xs, reports = batch.solve([B0, B1, ...])            # CUDA tensors (nrhs_k, n_k)
    """

    def __init__(self, matrices, nrhs, stream=None):
        L = _lib.load()
        self._mats = list(matrices)         # the handles must outlive the batch
        self.nrhs = [int(k) for k in nrhs]
        h = C.c_void_p()
        arr = (C.c_void_p * len(self._mats))(*[m._h for m in self._mats])
        cnt = (C.c_int * len(self.nrhs))(*self.nrhs)
        check(L.mf_batch_create(C.byref(h), len(self._mats), arr, cnt, C.c_void_p(stream) if stream else None),
              "mf_batch_create")
        self._h = h

    def tune(self, precision="mixed", iters=20, stream=None) -> int:
        cap = C.c_int()
        check(_lib.load().mf_batch_tune(self._h, _PREC[precision] if isinstance(precision, str) else precision,
                                        int(iters), C.byref(cap), C.c_void_p(stream) if stream else None),
              "mf_batch_tune")
        return cap.value

    def configure(self, cap, blocks_per_sm=1, stream=None) -> None:
        """Right-hand sides per work item and blocks per SM without timing runs
        (mf_batch_configure), e.g. a pair config() read after tune() on a batch
        of the same shapes."""
        check(_lib.load().mf_batch_configure(self._h, int(cap), int(blocks_per_sm),
                                             C.c_void_p(stream) if stream else None), "mf_batch_configure")

    def config(self):
        """(right-hand sides per item, blocks per SM) now in use (mf_batch_config)."""
        cap, lb = C.c_int(), C.c_int()
        check(_lib.load().mf_batch_config(self._h, C.byref(cap), C.byref(lb)), "mf_batch_config")
        return cap.value, lb.value

    def solve(self, Bs, Xs=None, options: Options | None = None, use_graph=True, stream=None, **kw):
        """Bs: CUDA float64 tensors of shape (nrhs_k, n_k).  Returns (Xs, reports)
        with reports[k] the list of system k's per-column report dicts."""
        import torch
        L = _lib.load()
        o = options if options is not None else default_options(**kw)
        Bs = [b.contiguous() for b in Bs]
        if Xs is None:
            Xs = [torch.zeros_like(b) for b in Bs]
        nb = len(Bs)
        pb = (C.c_void_p * nb)(*[b.data_ptr() for b in Bs])
        px = (C.c_void_p * nb)(*[x.data_ptr() for x in Xs])
        reps = (Report * sum(self.nrhs))()
        st = L.mf_batch_solve(self._h, pb, px, C.byref(o), reps, int(bool(use_graph)),
                              C.c_void_p(stream) if stream else None)
        flat = []
        for r in reps:
            d = r.as_dict()
            # batch reports: the column's work item's start / end after the
            # launch's first item start, and the blocks that solved it
            del d["phase_ms"]
            d["item_start_ms"], d["item_end_ms"], d["item_blocks"] = r.phase_ms[0], r.phase_ms[1], int(r.phase_ms[2])
            flat.append(d)
        out, k0 = [], 0
        for k in self.nrhs:
            out.append(flat[k0:k0 + k])
            k0 += k
        if st != _lib.MF_SUCCESS:
            err = MFError(st, "mf_batch_solve")
            err.report = out
            raise err
        return Xs, out

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().mf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_schedule(cost, tilem, grid: int):
    """The team sizes and list schedule a batch launch of `grid` blocks uses
    (mf_batch_schedule): (team per item, per-block lists of (item, rank),
    queue items largest first)."""
    L = _lib.load()
    n = len(cost)
    c = np.ascontiguousarray(cost, dtype=np.float64)
    t = np.ascontiguousarray(tilem, dtype=np.int32)
    team = np.zeros(max(n, 1), np.int32)
    bptr = np.zeros(grid + 1, np.int32)
    blist = np.zeros(2 * max(1, n * grid), np.int32)
    queue = np.zeros(max(n, 1), np.int32)
    nq = C.c_int()
    I = C.POINTER(C.c_int)
    check(L.mf_batch_schedule(n, c.ctypes.data_as(C.POINTER(C.c_double)), t.ctypes.data_as(I), int(grid),
                              team.ctypes.data_as(I), bptr.ctypes.data_as(I), blist.ctypes.data_as(I),
                              queue.ctypes.data_as(I), C.byref(nq)), "mf_batch_schedule")
    lists = [[(int(blist[2 * e]), int(blist[2 * e + 1])) for e in range(bptr[b], bptr[b + 1])] for b in range(grid)]
    return [int(v) for v in team[:n]], lists, [int(v) for v in queue[:nq.value]]


def read_matrix(path: str):
    """Reads .mtx / .cbd with the reference's semantics; returns
    (m, n, rowptr, colidx, val, is_symmetric) as numpy arrays."""
    L = _lib.load()
    m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rp, ci, vv = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    check(L.mf_read_matrix(path.encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp), C.byref(ci),
                           C.byref(vv), C.byref(sym)), f"mf_read_matrix({path})")
    rowptr = np.ctypeslib.as_array(rp, shape=(m.value + 1,)).copy()
    colidx = np.ctypeslib.as_array(ci, shape=(max(nnz.value, 1),))[: nnz.value].copy()
    val = np.ctypeslib.as_array(vv, shape=(max(nnz.value, 1),))[: nnz.value].copy()
    for p in (rp, ci, vv):
        L.mf_free_host(C.cast(p, C.c_void_p))
    return m.value, n.value, rowptr, colidx, val, bool(sym.value)


def write_cbd(path: str, m: int, n: int, rowptr, colidx, val) -> None:
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    colidx = np.ascontiguousarray(colidx, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    check(_lib.load().mf_write_cbd(path.encode(), int(m), int(n), int(colidx.size), _ptr(rowptr), _ptr(colidx),
                                   _ptr(val)), "mf_write_cbd")
