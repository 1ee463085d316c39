"""ctypes wrapper around oracle/liboracle.so (the CPU restatement) and, when it
was built, oracle/_ref/libmf_refhost.so (the reference's own host code).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference arm, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libmf_refhost.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")


class OrcTiles(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("tilem", "tilen", "tilenum", "csrsize", "csrptrlen")] + [
        ("tile_ptr", C.POINTER(C.c_int)), ("tile_columnidx", C.POINTER(C.c_int)),
        ("tile_nnz", C.POINTER(C.c_int)), ("blknnz", C.POINTER(C.c_int)),
        ("csr_offset", C.POINTER(C.c_int)), ("csrptr_offset", C.POINTER(C.c_int)),
        ("val", C.POINTER(C.c_double)), ("val_low", C.POINTER(C.c_float)),
        ("col", C.POINTER(C.c_ubyte)), ("ptr", C.POINTER(C.c_ubyte))]


class OrcRowlists(C.Structure):
    _fields_ = [("cnt", C.c_int), ("nonzero_row_new", C.POINTER(C.c_int)),
                ("blockrowid_new", C.POINTER(C.c_ubyte)), ("blockcsr_ptr_new", C.POINTER(C.c_ubyte)),
                ("tile_rowidx", C.POINTER(C.c_int)), ("block_signal", C.POINTER(C.c_int))]


class OrcOffsets(C.Structure):
    _fields_ = [("ptroffset1", C.POINTER(C.c_int)), ("ptroffset2", C.POINTER(C.c_int)),
                ("rowblkblock", C.c_int), ("blkcoostylerowidx", C.POINTER(C.c_uint)),
                ("colstart", C.POINTER(C.c_int)), ("colstop", C.POINTER(C.c_int))]


class OrcReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("relres_rec", C.c_double),
                ("relres_true", C.c_double), ("replacements", C.c_int)]


def build(ref_src: str | None = None) -> None:
    """Compile the oracle, and the reference-host harness when ref_src (the
    reference tree's src/ directory) is given."""
    cmd = ["make", "-s", "-C", HERE]
    if ref_src:
        cmd.append(f"REF_SRC={ref_src}")
    subprocess.run(cmd, check=True)


def _load():
    if not os.path.exists(_LIB):
        build()
    lib = C.CDLL(_LIB)
    lib.orc_tile_create.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f32p, C.POINTER(OrcTiles)]
    lib.orc_tiles_free.argtypes = [C.POINTER(OrcTiles)]
    lib.orc_offsets_build.argtypes = [C.POINTER(OrcTiles), C.c_int, C.POINTER(OrcOffsets)]
    lib.orc_offsets_free.argtypes = [C.POINTER(OrcOffsets)]
    lib.orc_rowlists_build.argtypes = [C.POINTER(OrcTiles), C.c_int, C.POINTER(OrcRowlists)]
    lib.orc_rowlists_free.argtypes = [C.POINTER(OrcRowlists)]
    lib.orc_encode_ref.argtypes = [C.c_int, _f64p, _f32p, _u16p, _i8p]
    lib.orc_encode_i8_scaled.argtypes = [C.POINTER(OrcTiles), _i8p, _f32p]
    lib.orc_f32_to_f16_rn.argtypes = [C.c_float]
    lib.orc_f32_to_f16_rn.restype = C.c_uint16
    lib.orc_classify_ref.argtypes = [C.c_double]
    lib.orc_segment_labels_ref.argtypes = [C.c_int, _f64p, _f64p, _i32p]
    lib.orc_spmv_tile.argtypes = [C.POINTER(OrcTiles), C.POINTER(OrcRowlists), C.c_int, _f64p, _f64p, C.c_int]
    for fn in (lib.orc_cg_fp64, lib.orc_bicgstab_fp64):
        fn.argtypes = [C.POINTER(OrcTiles), C.POINTER(OrcRowlists), C.c_int, _f64p, _f64p, C.c_double,
                       C.c_int, C.c_int, C.c_int, C.POINTER(OrcReport)]
    lib.orc_csr_spmv.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int]
    lib.orc_read_mtx.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_int)),
                                 C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int)]
    lib.orc_free.argtypes = [C.c_void_p]
    lib.orc_f64_to_f16_rn.argtypes = [C.c_double, C.c_double]
    lib.orc_f64_to_f16_rn.restype = C.c_uint16
    lib.orc_hfma.argtypes = [C.c_uint16, C.c_uint16, C.c_uint16]
    lib.orc_hfma.restype = C.c_uint16
    lib.orc_spmv_slices.argtypes = [C.POINTER(OrcTiles), C.c_int, _f64p, _f64p, C.c_int, _u16p, _i8p, _f32p]
    lib.orc_cg_parity.argtypes = [C.POINTER(OrcTiles), C.c_int, _f64p, _u16p, _i8p, _f64p, C.c_int, _i32p, _i32p,
                                  C.POINTER(OrcReport)]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _arr(ptr, n, dtype):
    if n <= 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


class Tiles:
    """Oracle tiling of a CSR matrix (Tile_create restated) plus the derived
    offsets and nonempty-row lists; keeps the C structures alive."""

    def __init__(self, rowA, colA, rowptr, colidx, val, val_low=None):
        L = lib()
        self.rowA, self.colA = int(rowA), int(colA)
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        if val_low is None:
            val_low = val.astype(np.float32)
        val_low = np.ascontiguousarray(val_low, dtype=np.float32)
        self.t = OrcTiles()
        if L.orc_tile_create(self.rowA, self.colA, rowptr, colidx, val, val_low, C.byref(self.t)) != 0:
            raise ValueError("orc_tile_create failed")
        self.o = OrcOffsets()
        L.orc_offsets_build(C.byref(self.t), self.rowA, C.byref(self.o))
        self.r = OrcRowlists()
        L.orc_rowlists_build(C.byref(self.t), self.rowA, C.byref(self.r))

    def __del__(self):
        try:
            L = lib()
            L.orc_tiles_free(C.byref(self.t))
            L.orc_offsets_free(C.byref(self.o))
            L.orc_rowlists_free(C.byref(self.r))
        except Exception:
            pass

    @property
    def dims(self):
        t = self.t
        return dict(tilem=t.tilem, tilen=t.tilen, tilenum=t.tilenum, csrsize=t.csrsize,
                    csrptrlen=t.csrptrlen, rowblkblock=self.o.rowblkblock, cnt_non_new=self.r.cnt)

    def arrays(self):
        t, o, r = self.t, self.o, self.r
        tm, tn = t.tilem, t.tilenum
        return {
            "tile_ptr": _arr(t.tile_ptr, tm + 1, np.int32),
            "tile_columnidx": _arr(t.tile_columnidx, tn, np.int32),
            "tile_nnz": _arr(t.tile_nnz, tn + 1, np.int32),
            "blknnz": _arr(t.blknnz, tn + 1, np.int32),
            "csr_offset": _arr(t.csr_offset, tn + 1, np.int32),
            "csrptr_offset": _arr(t.csrptr_offset, tn + 1, np.int32),
            "val": _arr(t.val, t.csrsize, np.float64),
            "val_low": _arr(t.val_low, t.csrsize, np.float32),
            "col": _arr(t.col, t.csrsize, np.uint8),
            "ptr": _arr(t.ptr, t.csrptrlen, np.uint8),
            "ptroffset1": _arr(o.ptroffset1, tn, np.int32),
            "ptroffset2": _arr(o.ptroffset2, tn, np.int32),
            "blkcoostylerowidx": _arr(o.blkcoostylerowidx, o.rowblkblock, np.uint32),
            "colstart": _arr(o.colstart, o.rowblkblock, np.int32),
            "colstop": _arr(o.colstop, o.rowblkblock, np.int32),
            "nonzero_row_new": _arr(r.nonzero_row_new, tn + 1, np.int32),
            "blockrowid_new": _arr(r.blockrowid_new, r.cnt + 1, np.uint8),
            "blockcsr_ptr_new": _arr(r.blockcsr_ptr_new, r.cnt + 1, np.uint8),
            "tile_rowidx": _arr(r.tile_rowidx, tn, np.int32),
            "block_signal": _arr(r.block_signal, tm + 4, np.int32),
        }

    def spmv_tile(self, x, nthreads=1):
        """The reference's host verification loop (uint8 end offsets included)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        need = max(self.t.tilen * 16, self.rowA)
        if x.size < need:
            x = np.concatenate([x, np.zeros(need - x.size)])
        y = np.zeros(max(self.t.tilem * 16, self.rowA), dtype=np.float64)
        lib().orc_spmv_tile(C.byref(self.t), C.byref(self.r), self.rowA, x, y, int(nthreads))
        return y[: self.rowA]

    def _solve(self, fn, b, tol, max_iter, fixed_iters, nthreads):
        if self.rowA % 16 == 1:
            # a one-row last tile-row has an empty payload in the reference layout
            raise ValueError("oracle solvers need rowA % 16 != 1 (reference one-row tile-row quirk)")
        b = np.ascontiguousarray(b[: self.rowA], dtype=np.float64)
        x = np.zeros(self.rowA, dtype=np.float64)
        rep = OrcReport()
        fn(C.byref(self.t), C.byref(self.r), self.rowA, b, x, float(tol), int(max_iter),
           int(bool(fixed_iters)), int(nthreads), C.byref(rep))
        return x, dict(iterations=rep.iterations, converged=bool(rep.converged),
                       relres_rec=rep.relres_rec, relres_true=rep.relres_true,
                       replacements=rep.replacements)

    def _encoded(self):
        """The reference encoder's FP16 / truncated INT8 values and this
        build's scaled INT8 values, in tile payload order (cached)."""
        if not hasattr(self, "_enc"):
            a = self.arrays()
            f16, i8ref = encode_ref(a["val"], a["val_low"])
            q8, sc = encode_i8_scaled(self)
            pad = lambda v, dt: np.ascontiguousarray(v if v.size else np.zeros(1, dt), dtype=dt)
            self._enc = (pad(f16, np.uint16), pad(i8ref, np.int8), pad(q8, np.int8), pad(sc, np.float32))
        return self._enc

    def spmv_slices(self, x, prec):
        """y = A x with every tile's values stored in one precision (0 FP64,
        1 FP32, 2 FP16, 3 scaled INT8), FP64 accumulation in the GPU slice
        walk's entry order (orc_spmv_slices)."""
        f16, _, q8, sc = self._encoded()
        x = np.ascontiguousarray(x, dtype=np.float64)
        need = max(self.t.tilen * 16, self.rowA)
        if x.size < need:
            x = np.concatenate([x, np.zeros(need - x.size)])
        y = np.zeros(max(self.t.tilem * 16, self.rowA, 1), dtype=np.float64)
        lib().orc_spmv_slices(C.byref(self.t), self.rowA, x, y, int(prec), f16, q8, sc)
        return y[: self.rowA]

    def cg_parity(self, b, iters):
        """The reference's mixed CG (parity arithmetic and label rule) for
        `iters` fixed iterations from x0 = 0 (orc_cg_parity).  Returns (x,
        labels of the next SpMV per column segment, all-lanes-agree mask,
        report)."""
        f16, i8ref, _, _ = self._encoded()
        b = np.ascontiguousarray(b[: self.rowA], dtype=np.float64)
        x = np.zeros(self.rowA, dtype=np.float64)
        nseg = max(self.t.tilen, 1)
        labels = np.zeros(nseg, dtype=np.int32)
        agree = np.zeros(nseg, dtype=np.int32)
        rep = OrcReport()
        lib().orc_cg_parity(C.byref(self.t), self.rowA, b, f16, i8ref, x, int(iters), labels, agree, C.byref(rep))
        return x, labels[: self.t.tilen], agree[: self.t.tilen].astype(bool), dict(
            iterations=rep.iterations, relres_rec=rep.relres_rec, relres_true=rep.relres_true)

    def cg_fp64(self, b, tol=1e-8, max_iter=10000, fixed_iters=False, nthreads=1):
        return self._solve(lib().orc_cg_fp64, b, tol, max_iter, fixed_iters, nthreads)

    def bicgstab_fp64(self, b, tol=1e-8, max_iter=10000, fixed_iters=False, nthreads=1):
        return self._solve(lib().orc_bicgstab_fp64, b, tol, max_iter, fixed_iters, nthreads)


def encode_ref(val, val_low=None):
    val = np.ascontiguousarray(val, dtype=np.float64)
    if val_low is None:
        val_low = val.astype(np.float32)
    val_low = np.ascontiguousarray(val_low, dtype=np.float32)
    f16 = np.zeros(val.size, dtype=np.uint16)
    i8 = np.zeros(val.size, dtype=np.int8)
    lib().orc_encode_ref(val.size, val, val_low, f16, i8)
    return f16, i8


def encode_i8_scaled(tiles: Tiles):
    q = np.zeros(max(tiles.t.csrsize, 1), dtype=np.int8)
    s = np.zeros(max(tiles.t.tilenum, 1), dtype=np.float32)
    lib().orc_encode_i8_scaled(C.byref(tiles.t), q, s)
    return q[: tiles.t.csrsize], s[: tiles.t.tilenum]


def f64_to_f16_rn(s, e=0.0):
    return int(lib().orc_f64_to_f16_rn(float(s), float(e)))


def hfma(a, b, c):
    """__hfma on binary16 bit patterns (orc_hfma)."""
    return int(lib().orc_hfma(int(a), int(b), int(c)))


def segment_labels_ref(p_old, p_new):
    p_old = np.ascontiguousarray(p_old, dtype=np.float64)
    p_new = np.ascontiguousarray(p_new, dtype=np.float64)
    nseg = p_old.size // 16
    vis = np.zeros(max(nseg, 1), dtype=np.int32)
    lib().orc_segment_labels_ref(nseg, p_old, p_new, vis)
    return vis[:nseg]


def csr_spmv(rowptr, colidx, val, x, n=None, nthreads=1):
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    n = rowptr.size - 1 if n is None else n
    y = np.zeros(n, dtype=np.float64)
    lib().orc_csr_spmv(n, rowptr, np.ascontiguousarray(colidx, dtype=np.int32),
                       np.ascontiguousarray(val, dtype=np.float64),
                       np.ascontiguousarray(x, dtype=np.float64), y, int(nthreads))
    return y


def read_mtx(path):
    L = lib()
    m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rp, ci, vv = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    rc = L.orc_read_mtx(path.encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp),
                        C.byref(ci), C.byref(vv), C.byref(sym))
    if rc != 0:
        raise IOError(f"orc_read_mtx({path}) failed: {rc}")
    out = (m.value, n.value, _arr(rp, m.value + 1, np.int32), _arr(ci, nnz.value, np.int32),
           _arr(vv, nnz.value, np.float64), bool(sym.value))
    for p in (rp, ci, vv):
        L.orc_free(C.cast(p, C.c_void_p))
    return out


# ---------------------------------------------------------------- reference host code

def ref_available() -> bool:
    return os.path.exists(_REF)


_ref = None


def _reflib():
    global _ref
    if _ref is None:
        r = C.CDLL(_REF)
        r.ref_tile_create.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f32p]
        r.ref_tile_create.restype = C.c_void_p
        r.ref_tile_dims.argtypes = [C.c_void_p, _i32p]
        r.ref_tile_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        r.ref_tile_free.argtypes = [C.c_void_p]
        r.ref_read_matrix.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_int)),
                                      C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_double)),
                                      C.POINTER(C.c_int)]
        r.ref_free.argtypes = [C.c_void_p]
        _ref = r
    return _ref


def ref_tile_create(rowA, colA, rowptr, colidx, val, val_low=None):
    """Run the reference's own Tile_create + blockspmv_cpu offsets."""
    r = _reflib()
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    colidx = np.ascontiguousarray(colidx, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    if val_low is None:
        val_low = val.astype(np.float32)
    val_low = np.ascontiguousarray(val_low, dtype=np.float32)
    nnz = int(rowptr[-1])
    h = r.ref_tile_create(int(rowA), int(colA), nnz, rowptr, colidx, val, val_low)
    d = np.zeros(6, dtype=np.int32)
    r.ref_tile_dims(h, d)
    tm, tn, cs, cpl, rb = int(d[0]), int(d[2]), int(d[3]), int(d[4]), int(d[5])
    spec = {"tile_ptr": (tm + 1, np.int32), "tile_columnidx": (tn, np.int32),
            "tile_nnz": (tn + 1, np.int32), "blknnz": (tn + 1, np.int32),
            "csr_offset": (tn + 1, np.int32), "csrptr_offset": (tn + 1, np.int32),
            "val": (cs, np.float64), "val_low": (cs, np.float32), "col": (cs, np.uint8),
            "ptr": (cpl, np.uint8), "ptroffset1": (tn, np.int32), "ptroffset2": (tn, np.int32),
            "blkcoostylerowidx": (rb, np.uint32), "colstart": (rb, np.int32), "colstop": (rb, np.int32)}
    out = {}
    for k, (n, dt) in spec.items():
        a = np.zeros(max(n, 1), dtype=dt)
        if r.ref_tile_get(h, k.encode(), a.ctypes.data_as(C.c_void_p)) != 0:
            raise KeyError(k)
        out[k] = a[:n]
    r.ref_tile_free(h)
    dims = dict(tilem=tm, tilen=int(d[1]), tilenum=tn, csrsize=cs, csrptrlen=cpl, rowblkblock=rb)
    return dims, out


def ref_read_matrix(path):
    r = _reflib()
    m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rp, ci, vv = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    r.ref_read_matrix(path.encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp),
                      C.byref(ci), C.byref(vv), C.byref(sym))
    out = (m.value, n.value, _arr(rp, m.value + 1, np.int32), _arr(ci, nnz.value, np.int32),
           _arr(vv, nnz.value, np.float64), bool(sym.value))
    for p in (rp, ci, vv):
        r.ref_free(C.cast(p, C.c_void_p))
    return out
