"""One fixed set of library calls, run through whichever build the
MILLEFEUILLE_LIB environment variable names (the normal libmillefeuille.so or
the bounds-checked libmillefeuille_check.so), with every result saved, so that
a test can compare the two builds bit for bit:

    MILLEFEUILLE_LIB=<lib> python tests/harness/check_run.py OUT.npz
    MILLEFEUILLE_LIB=<lib> python tests/harness/check_run.py OUT.npz --narrowed

The calls cover every kernel the bounds checks sit in: the persistent solve
(FP64, mixed, parity CG; mixed BiCGSTAB), the standalone SpMV (FP64, FP32 and
each stored precision), several right-hand sides, a batch with a dynamic queue
and a team item (with and without graph replay), the 8-column SpMM on the CUDA
and the tensor cores, and the allocation-free SpMV.

--narrowed runs one mixed CG with the test_check_limit hook: the kernels check
the operand's gathered entries against a length shorter than the vector, so
gathers past it fail their check (every access stays inside the real vector;
the failing ones are skipped).  The solve must return MF_ERR_CHECK, and a
normal solve on the same context right after it must succeed.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "mille-feuille_b200"))


def run_all(mf, M, torch):
    res = {}
    A, b, _ = M.poisson3d_varcoef(16, seed=1)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    for prec in ("fp64", "mixed"):
        x, r = G.solve(b, method="cg", precision=prec, tol=1e-10 if prec == "fp64" else 1e-8)
        res[f"cg_{prec}"], res[f"cg_{prec}_it"] = x, r["iterations"]
    x, r = G.solve(b * 1e-6, method="cg", precision="parity", max_iter=20, fixed_iters=1, replace_every=0)
    res["cg_parity"], res["cg_parity_labels"] = x, G.solver_labels()
    C, bc, _ = M.convdiff3d(12, seed=2)
    Gc = mf.Matrix.from_csr(C.n, C.n, C.rowptr, C.colidx, C.val)
    x, r = Gc.solve(bc, method="bicgstab", precision="mixed", tol=1e-8)
    res["bicgstab_mixed"], res["bicgstab_mixed_it"] = x, r["iterations"]
    # a wide random matrix: tile-rows spanning several slices, a ragged last tile-row
    W = M.random_csr(500, 530, 0.06, seed=4)
    Gw = mf.Matrix.from_csr(W.n, 530, W.rowptr, W.colidx, W.val)
    xw = np.random.default_rng(11).uniform(-1, 1, 530)
    for p in range(4):
        res[f"spmv_tiles_{p}"] = Gw.spmv_tiles(xw, p)
    xs = np.random.default_rng(12).uniform(-1, 1, A.n)
    res["spmv_fp64"] = G.spmv(xs, precision="fp64")
    res["spmv_mixed"] = G.spmv(xs, precision="mixed")
    B3 = np.stack([b, np.roll(b, 5), np.random.default_rng(13).uniform(-1, 1, A.n)])
    for prec in ("fp64", "mixed"):
        X, reps = G.solve_multi(B3, method="cg", precision=prec, tol=1e-8)
        res[f"multi_{prec}"] = X
    # batch: small queue items and one larger system
    mats, Bs = [], []
    for k, (_, _, S, Bk) in enumerate(M.batch_systems(6, seed=3, side2d=(8, 40), side3d=(4, 10), rhs=(1, 4))):
        mats.append(mf.Matrix.from_csr(S.n, S.n, S.rowptr, S.colidx, S.val))
        Bs.append(torch.from_numpy(Bk).cuda())
    L2, bl, _ = M.poisson3d_varcoef(40, seed=5)
    mats.append(mf.Matrix.from_csr(L2.n, L2.n, L2.rowptr, L2.colidx, L2.val))
    Bs.append(torch.from_numpy(bl[None, :].copy()).cuda())
    batch = mf.Batch(mats, [t.shape[0] for t in Bs])
    for graph in (False, True):
        Xs, reps = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=graph)
        for k, X in enumerate(Xs):
            res[f"batch_g{int(graph)}_{k}"] = X.cpu().numpy()
        res[f"batch_g{int(graph)}_blocks"] = np.array([rk[0]["item_blocks"] for rk in reps])
    batch.close()
    Sa = M.aniso2d_grf(64, seed=4, nrhs=1)[0]
    Ga = mf.Matrix.from_csr(Sa.n, Sa.n, Sa.rowptr, Sa.colidx, Sa.val)
    X8 = np.random.default_rng(14).uniform(-1, 1, (8, Ga.info["n_cols"]))
    for tc in (False, True):
        res[f"spmm8_tc{int(tc)}"] = Ga.spmm8(X8, tensor_cores=tc)[0]
    xd = torch.from_numpy(xs).cuda()
    yd = torch.empty_like(xd)
    G.spmv_noalloc(xd, yd, precision="fp64")
    torch.cuda.synchronize()
    res["spmv_noalloc"] = yd.cpu().numpy()
    # a synchronous call after the asynchronous one reports any check it failed
    res["spmv_after_noalloc"] = G.spmv(xs, precision="fp64")
    return res


def run_narrowed(mf, M):
    A, b, _ = M.poisson3d_varcoef(16, seed=1)
    G = mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val)
    status = 0
    try:
        G.solve(b, method="cg", precision="mixed", tol=1e-8, max_iter=5, test_check_limit=A.n // 2)
    except mf.MFError as e:
        status = e.status
    x, r = G.solve(b, method="cg", precision="mixed", tol=1e-8)
    return {"narrowed_status": status, "after_converged": int(r["converged"]), "after_relres": r["relres_true"]}


def main():
    import torch
    import millefeuille as mf
    from millefeuille import matrices as M
    out = sys.argv[1]
    torch.cuda.set_device(0)
    res = {"arch": mf._lib.load().mf_build_arch().decode()}
    if "--narrowed" in sys.argv:
        res.update(run_narrowed(mf, M))
    else:
        res.update(run_all(mf, M, torch))
    np.savez(out, **{k: np.asarray(v) for k, v in res.items()})


if __name__ == "__main__":
    main()
