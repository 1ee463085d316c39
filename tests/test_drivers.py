"""The drop-in benchmark executables (bin/main-cg, main-cg-mixed, main-bicg,
main-bicg-mixed): command lines, prints and CSV rows of the reference's
drivers (main-cg.cu:1682-1764, main-cg-mixed.cu:3071-3144,
main-bicg-mixed.cu:2168-2193), checked against the library's own solve."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "mille-feuille_b200", "bin")
NAMES = ["main-cg", "main-cg-mixed", "main-bicg", "main-bicg-mixed"]


@pytest.fixture(scope="module")
def drivers(mf):
    import importlib
    importlib.import_module("build").build_drivers()
    return {n: os.path.join(BIN, n) for n in NAMES}


def test_drivers_print_usage_without_arguments(drivers):
    for name, exe in drivers.items():
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 1 and r.stderr.startswith(f"usage: {name} ")


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["cg", "cg_mixed"])
def test_cg_driver_writes_reference_csv_row(mf, cuda, drivers, tmp_path, variant):
    from millefeuille import matrices as M
    A, _, _ = M.poisson3d_varcoef(16, seed=1)
    mtx = str(tmp_path / "p16.mtx")
    M.write_mtx(mtx, A)
    csv = str(tmp_path / "out.csv")
    exe = drivers["main-cg" if variant == "cg" else "main-cg-mixed"]
    for _ in range(2):                       # second run appends, no second header
        r = subprocess.run([exe, mtx, "30", csv], capture_output=True, text=True, cwd=tmp_path)
        assert r.returncode == 0, r.stderr
    tag = "time_cg_avg=" if variant == "cg" else "time_cg-mixed_avg="
    assert tag in r.stdout and "(warmup=3, benchmark=10)" in r.stdout
    lines = open(csv).read().splitlines()
    assert lines[0] == "matrix,variant,iterations,time_ms,nnz,l2_norm,residual" and len(lines) == 3
    f = lines[2].split(",")
    assert f[0] == mtx and f[1] == variant and int(f[2]) == 30 and int(f[4]) == A.nnz
    # the residual column against the library's own solve of b = A 1 with 30 fixed
    # iterations; b summed in entry order like the driver: after ~30 iterations CG
    # amplifies even a one-ulp difference in b into a visibly different residual
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    b = np.zeros(A.n)
    for i in range(A.n):
        s = 0.0
        for j in range(A.rowptr[i], A.rowptr[i + 1]):
            s += A.val[j]
        b[i] = s
    _, rep = G.solve(b, method="cg", precision="fp64" if variant == "cg" else "mixed", max_iter=30,
                     fixed_iters=1, replace_every=0)
    assert float(f[5]) == pytest.approx(rep["relres_true"], rel=1e-5)


@pytest.mark.gpu
def test_bicg_driver_appends_its_row(mf, cuda, drivers, tmp_path):
    from millefeuille import matrices as M
    A, _, _ = M.convdiff3d(16, seed=2)
    mtx = str(tmp_path / "cd16.mtx")
    M.write_mtx(mtx, A)
    r = subprocess.run([drivers["main-bicg-mixed"], mtx], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "time_bicg=" in r.stdout
    rows = open(tmp_path / "bicg_mixed_performance.csv").read().splitlines()
    assert len(rows) == 1 and rows[0].startswith(mtx + ",")
