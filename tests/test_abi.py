"""CPU tests of the C ABI: the library loads, exports every symbol the header
declares, and its host-only entry points (status strings, options, matrix
reader / writer) behave; no compute call is made without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def _declared_functions():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?[\s\*])([A-Za-z_]\w*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof", "defined"):
                names.add(name)
    return sorted(names)


def test_library_exports_every_declared_symbol(mf):
    from millefeuille import _lib
    L = _lib.load()
    declared = _declared_functions()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) <= set(declared)


def test_status_strings_and_defaults(mf):
    from millefeuille import _lib
    L = _lib.load()
    assert L.mf_build_arch().decode() == "sm_100a"
    for s in range(0, 10):
        assert len(_lib.status_string(s)) > 3
    o = mf.default_options()
    assert o.precision == mf.MF_PREC_MIXED and o.replace_every == 50 and o.tol == 1e-8
    o2 = mf.default_options(precision="fp64", method="bicgstab", tol=1e-10)
    assert o2.precision == 0 and o2.method == 1 and o2.tol == 1e-10
    # the ctypes mirror of mf_options has the C layout: the last field is set by mf_options_default
    assert o.demote_min_fraction == 0.125 and o.x0_given == 0 and o.l2_window == 1 and o.use_lossless == 1
    assert o.demote_fp16 == 2.0 ** -13 and o.demote_int8 == 2.0 ** -16 and o.wait_timeout_s == 10.0


def test_checked_build_loads_and_exports_the_same_symbols(mf):
    """libmillefeuille_check.so (build.py --check) has the normal build's ABI."""
    from millefeuille import _lib
    if not os.path.exists(_lib.LIB_CHECK_PATH):
        import importlib
        importlib.import_module("build").build(check=True)
    L = C.CDLL(_lib.LIB_CHECK_PATH)
    missing = [n for n in _declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    L.mf_build_arch.restype = C.c_char_p
    assert L.mf_build_arch().decode() == "sm_100a (bounds-checked)"
    L.mf_status_string.restype = C.c_char_p
    assert b"bounds check" in L.mf_status_string(9)
    o = _lib.Options()
    L.mf_options_default(C.byref(o))
    assert o.test_check_limit == 0 and o.relax_int8 == 0 and o.demote_min_fraction == 0.125


def test_no_device_reports_not_built(mf):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(mf.MFError) as e:
        mf.Matrix.from_csr(2, 2, np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, 1.0]))
    assert e.value.status == 8


@pytest.mark.parametrize("field,sym", [("real", False), ("real", True), ("pattern", False), ("integer", True)])
def test_mtx_reader_matches_oracle_and_reference(mf, oracle_mod, tmp_path, field, sym):
    from millefeuille import matrices as M
    A = M.random_csr(70, 70, 0.08, seed=5)
    S = A.to_scipy()
    if sym:
        S = (S + S.T).tocsr()
        S.sort_indices()
        A = M.CSR(70, S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data * 3.0)
    if field == "integer":
        A.val = np.round(A.val * 10)
    path = str(tmp_path / "m.mtx")
    M.write_mtx(path, A, symmetric=sym, field=field)
    got = mf.read_matrix(path)
    exp = oracle_mod.read_mtx(path)
    for g, e in zip(got[2:5], exp[2:5]):
        np.testing.assert_array_equal(g, e)
    assert got[:2] == exp[:2] and got[5] == exp[5]
    if oracle_mod.ref_available():
        ref = oracle_mod.ref_read_matrix(path)
        for g, e in zip(got[2:5], ref[2:5]):
            np.testing.assert_array_equal(g, e)


@pytest.mark.parametrize("sym", [False, True])
def test_mtx_reader_parallel_chunks_keep_file_order(mf, oracle_mod, tmp_path, sym):
    """A file of several MB is parsed in line-aligned chunks by several host
    threads; entries shuffled in the file (and mirrored ones) must land in
    file order within each row, as the serial oracle places them."""
    rng = np.random.default_rng(12)
    n, nz = 20000, 300000
    r = rng.integers(1, n + 1, nz)
    c = rng.integers(1, n + 1, nz)
    if sym:
        r, c = np.maximum(r, c), np.minimum(r, c)
    v = rng.standard_normal(nz)
    path = tmp_path / "big.mtx"
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {'symmetric' if sym else 'general'}\n")
        f.write("% comment line\n")
        f.write(f"{n} {n} {nz}\n")
        f.write("".join(f"{a} {b} {x!r}\n" for a, b, x in zip(r.tolist(), c.tolist(), v.tolist())))
    assert path.stat().st_size > 4 << 20
    got = mf.read_matrix(str(path))
    exp = oracle_mod.read_mtx(str(path))
    assert got[:2] == exp[:2] and got[5] == exp[5]
    for g, e in zip(got[2:5], exp[2:5]):
        np.testing.assert_array_equal(g, e)


def test_cbd_roundtrip(mf, tmp_path):
    from millefeuille import matrices as M
    A = M.random_csr(50, 60, 0.1, seed=6)
    p = str(tmp_path / "a.cbd")
    mf.write_cbd(p, 50, 60, A.rowptr, A.colidx, A.val)
    m, n, rp, ci, vv, sym = mf.read_matrix(p)
    assert (m, n) == (50, 60)
    np.testing.assert_array_equal(rp, A.rowptr)
    np.testing.assert_array_equal(ci, A.colidx)
    np.testing.assert_array_equal(vv, A.val)
    p2 = str(tmp_path / "b.cbd")
    M.write_cbd(p2, A, ncols=60)
    assert open(p, "rb").read() == open(p2, "rb").read()


def test_reader_rejects_bad_files(mf, tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    with pytest.raises(mf.MFError):
        mf.read_matrix(str(p))
    with pytest.raises(mf.MFError):
        mf.read_matrix(str(tmp_path / "missing.mtx"))
