"""The reference's main-cg dispatch relinked against this library: a C
program written against main-cg.cu's entry points (tests/harness/
main_cg_dispatch.c; nnz < 10,000 -> cg_solve_inc) is built against
libmillefeuille_fp64.so, where cg_solve_inc is main-cg.cu's FP64 solver, and
against libmillefeuille.so, where it is main-cg-mixed.cu's mixed solver.  The
library's record of the solve (mf_dropin_last_report) shows which precision
ran; the FP64 build's l2_norm equals the FP64 oracle's residual after the same
fixed iteration count (rel 1e-9: the summation order differs)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mille-feuille_b200", "millefeuille")
SRC = os.path.join(ROOT, "tests", "harness", "main_cg_dispatch.c")


def _build(tmp_path, lib):
    exe = str(tmp_path / f"dispatch_{lib}")
    cmd = ["gcc", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe, "-L", PKG, f"-l{lib}",
           f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_dispatch_harness_builds_against_both_libraries(mf, tmp_path):
    for lib in ("millefeuille", "millefeuille_fp64"):
        exe = _build(tmp_path, lib)
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 1 and "usage" in r.stderr


@pytest.mark.gpu
def test_relinked_main_cg_dispatch_runs_fp64_cg_solve_inc(mf, oracle_mod, cuda, tmp_path):
    import numpy as np
    from millefeuille import matrices as M
    A = M.laplace2d(40)                      # nnz = 7,840 < 10,000: main-cg calls cg_solve_inc
    assert A.nnz < 10000
    mtx = str(tmp_path / "lap40.mtx")
    M.write_mtx(mtx, A)
    out = {}
    for lib in ("millefeuille_fp64", "millefeuille"):
        r = subprocess.run([_build(tmp_path, lib), mtx, "25"], capture_output=True, text=True, cwd=tmp_path)
        assert r.returncode == 0, r.stderr
        kv = dict(t.split("=", 1) for t in r.stdout.split()[:4])
        out[lib] = kv
        assert kv["entry"] == "cg_solve_inc" and int(kv["iterations"]) == 25
    t64 = [int(v) for v in out["millefeuille_fp64"]["tiles"].split(",")]
    tmx = [int(v) for v in out["millefeuille"]["tiles"].split(",")]
    assert t64[0] > 0 and t64[1] == t64[2] == t64[3] == 0, t64        # FP64 tiles only
    assert tmx[0] == 0 and sum(tmx[1:]) > 0, tmx                      # the mixed solver
    b = A.matvec(np.ones(A.n))
    T = oracle_mod.Tiles(A.n, A.n, A.rowptr, A.colidx, A.val)
    _, ro = T.cg_fp64(b, max_iter=25, fixed_iters=True)
    assert float(out["millefeuille_fp64"]["l2_norm"]) == pytest.approx(ro["relres_true"], rel=1e-9)
