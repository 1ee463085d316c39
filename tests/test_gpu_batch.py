"""Batched solves (mf_batch_*): many uneven systems with 1 - 16 right-hand
sides each in one persistent launch, against single-system solves.

Tolerances: every column converges on its own FP64 true residual; columns
agree with single-system solves to 1e-7 of max|x| at tol 1e-10 (same
algorithm, block-level instead of grid-level reduction order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems():
    from millefeuille import matrices as M
    return M.batch_systems(14, seed=3, side2d=(8, 48), side3d=(4, 12), rhs=(1, 16))


def _relres(A, x, b):
    return np.linalg.norm(A.to_scipy() @ x - b) / np.linalg.norm(b)


def _setup(mf, systems):
    import torch
    mats = [mf.Matrix.from_csr(A.n, A.n, A.rowptr, A.colidx, A.val) for _, _, A, _ in systems]
    Bs = [torch.from_numpy(B).cuda() for _, _, _, B in systems]
    return mats, Bs


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-8)])
def test_batch_converges_and_matches_single_solves(mf, cuda, systems, precision, tol):
    mats, Bs = _setup(mf, systems)
    batch = mf.Batch(mats, [B.shape[0] for B in Bs])
    Xs, reps = batch.solve(Bs, method="cg", precision=precision, tol=tol, use_graph=False)
    for (kind, side, A, B), X, rk, G in zip(systems, Xs, reps, mats):
        X = X.cpu().numpy()
        assert len(rk) == B.shape[0]
        for c in range(B.shape[0]):
            assert rk[c]["converged"] and rk[c]["relres_true"] <= tol, (kind, side, c, rk[c])
            assert _relres(A, X[c], B[c]) <= tol * 1.0001
        if precision == "fp64":
            xs, _ = G.solve(B[0], method="cg", precision="fp64", tol=tol)
            np.testing.assert_allclose(X[0], xs, rtol=0, atol=1e-7 * np.abs(xs).max())


def test_batch_graph_replay_and_tuning(mf, cuda, systems):
    import torch
    mats, Bs = _setup(mf, systems)
    batch = mf.Batch(mats, [B.shape[0] for B in Bs])
    X0, r0 = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=False)
    Xg, rg = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=True)    # capture + run
    Xs = [torch.full_like(b, 7.0) for b in Bs]
    Xs, rr = batch.solve(Bs, Xs, method="cg", precision="mixed", tol=1e-8, use_graph=True)  # new X: recapture
    Xs2, rr2 = batch.solve(Bs, Xs, method="cg", precision="mixed", tol=1e-8, use_graph=True)  # replay
    for a, b, c, d in zip(X0, Xg, Xs, Xs2):
        assert torch.equal(a, b) and torch.equal(a, c) and torch.equal(a, d)     # deterministic
    assert [[x["iterations"] for x in s] for s in r0] == [[x["iterations"] for x in s] for s in rr2]
    cap = batch.tune("mixed", iters=10)
    assert cap in (2, 4, 8)
    Xt, rt = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8)
    for (kind, side, A, B), X, rk in zip(systems, Xt, rt):
        for c in range(B.shape[0]):
            assert rk[c]["converged"] and _relres(A, X.cpu().numpy()[c], B[c]) <= 1.0001e-8
    # the tuned pair, read back and given to a new batch of the same systems
    # without timing runs: the same items and kernels, the same bits
    cfg = batch.config()
    assert cfg[0] == cap and cfg[1] in (1, 2)
    for bad in ((3, 1), (0, 1), (8, 2), (4, 3)):
        with pytest.raises(mf.MFError):
            batch.configure(*bad)
    assert batch.config() == cfg
    other = mf.Batch(mats, [B.shape[0] for B in Bs])
    other.configure(*cfg)
    Xo, ro = other.solve(Bs, method="cg", precision="mixed", tol=1e-8)
    assert other.config() == cfg
    for a, b in zip(Xt, Xo):
        assert torch.equal(a, b)
    assert rt[0][0]["grid_blocks"] == ro[0][0]["grid_blocks"]
    other.close()


def test_batch_rejects_bad_input(mf, cuda, systems):
    mats, Bs = _setup(mf, systems[:2])
    with pytest.raises(mf.MFError):
        mf.Batch(mats, [0, 1])
    batch = mf.Batch(mats, [B.shape[0] for B in Bs])
    with pytest.raises(mf.MFError) as e:
        batch.solve(Bs, method="bicgstab")
    assert e.value.status == 5


def test_batch_split_over_parts_matches_one_batch(mf, cuda, systems):
    """The multi-GPU split run part by part on one GPU (each part its own
    mf_batch, as each rank would): every system converges and agrees with the
    single batch (a part may give an item a different team size, so the
    reduction order, and with it the last digits, can differ)."""
    from millefeuille import shard
    mats, Bs = _setup(mf, systems)
    nr = [B.shape[0] for B in Bs]
    X1, r1 = mf.Batch(mats, nr).solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=False)
    part, _ = shard.partition([A.n for _, _, A, _ in systems], [A.nnz for _, _, A, _ in systems], nr, 3)
    for q in range(3):
        own = shard.owned(part, q)
        assert own
        Xq, rq = mf.Batch([mats[k] for k in own], [nr[k] for k in own]).solve(
            [Bs[k] for k in own], method="cg", precision="mixed", tol=1e-8, use_graph=False)
        for k, X, rk in zip(own, Xq, rq):
            A, B = systems[k][2], systems[k][3]
            x1 = X1[k].cpu().numpy()
            x = X.cpu().numpy()
            for c in range(B.shape[0]):
                assert rk[c]["converged"] and _relres(A, x[c], B[c]) <= 1.0001e-8
            np.testing.assert_allclose(x, x1, rtol=0, atol=1e-4 * np.abs(x1).max())


def test_batch_team_items(mf, cuda):
    """An item far above a fair share of the launch (one 27-point system of
    64,000 unknowns with 8 right-hand sides next to small ones) is solved by a
    team of blocks: every column converges on its FP64 true residual, the large
    system agrees with a single-system FP64 solve, and a replay from a CUDA
    graph (a cooperative launch in the graph) is bitwise the direct launch."""
    import torch
    from millefeuille import matrices as M
    big = M.batch_systems(1, seed=11, side2d=(256, 256), side3d=(40, 40), rhs=(8, 8))
    small = M.batch_systems(6, seed=12, side2d=(8, 24), side3d=(4, 8), rhs=(1, 4))
    systems = big + small
    mats, Bs = _setup(mf, systems)
    batch = mf.Batch(mats, [B.shape[0] for B in Bs])
    X0, r0 = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=False)
    Xg, rg = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=True)
    Xh, rh = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=True)
    for a, b, c in zip(X0, Xg, Xh):
        assert torch.equal(a, b) and torch.equal(a, c)
    assert r0[0][0]["grid_blocks"] > 1
    for (kind, side, A, B), X, rk, G in zip(systems, X0, r0, mats):
        X = X.cpu().numpy()
        for c in range(B.shape[0]):
            assert rk[c]["converged"] and _relres(A, X[c], B[c]) <= 1.0001e-8, (kind, side, c, rk[c])
    xs, _ = mats[0].solve(systems[0][3][0], method="cg", precision="fp64", tol=1e-12)
    np.testing.assert_allclose(X0[0].cpu().numpy()[0], xs, rtol=0, atol=1e-5 * np.abs(xs).max())


def test_batch_team_wait_timeout_is_reported(mf, cuda):
    """Failure detection on the team path without a GPU fault: with the test
    hook every team's first barrier waits for an arrival that never comes; the
    bounded wait gives up after wait_timeout_s, the batch returns
    MF_ERR_TIMEOUT, and the same batch then solves normally (the context stays
    usable)."""
    from millefeuille import matrices as M
    systems = M.batch_systems(1, seed=11, side2d=(256, 256), side3d=(40, 40), rhs=(8, 8)) + \
        M.batch_systems(3, seed=12, side2d=(8, 24), side3d=(4, 8), rhs=(1, 4))
    mats, Bs = _setup(mf, systems)
    batch = mf.Batch(mats, [B.shape[0] for B in Bs])
    o = mf.default_options(precision="mixed", tol=1e-8, wait_timeout_s=0.5, test_stall_barrier=1)
    with pytest.raises(mf.MFError) as e:
        batch.solve(Bs, options=o, use_graph=False)
    assert e.value.status == 4                      # MF_ERR_TIMEOUT
    assert e.value.report[0][0]["item_blocks"] > 1
    X, r = batch.solve(Bs, method="cg", precision="mixed", tol=1e-8, use_graph=False)
    for (kind, side, A, B), Xk, rk in zip(systems, X, r):
        Xk = Xk.cpu().numpy()
        for c in range(B.shape[0]):
            assert rk[c]["converged"] and _relres(A, Xk[c], B[c]) <= 1.0001e-8


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-8)])
def test_batch_initial_guess(mf, cuda, systems, precision, tol):
    """x0_given: every column starts from the X passed in (R = B - A X formed in
    FP64 inside the launch).  From converged solutions no iteration runs; from
    a 20-iteration start every column converges in fewer iterations than from
    zero and to the same tolerance, with and without graph replay."""
    mats, Bs = _setup(mf, systems)
    batch = mf.Batch(mats, [B.shape[0] for B in Bs])
    X1, r1 = batch.solve(Bs, method="cg", precision="fp64", tol=1e-10, use_graph=False)
    X2, r2 = batch.solve(Bs, [x.clone() for x in X1], method="cg", precision=precision, tol=tol, x0_given=1,
                         use_graph=False)
    for rk in r2:
        for col in rk:
            assert col["converged"] and col["iterations"] <= 1, col
    Xh, _ = batch.solve(Bs, method="cg", precision="fp64", max_iter=20, fixed_iters=1, use_graph=False)
    for graph in (False, True):
        X3, r3 = batch.solve(Bs, [x.clone() for x in Xh], method="cg", precision=precision, tol=tol, x0_given=1,
                             use_graph=graph)
        for (kind, side, A, B), X, rk, rk0 in zip(systems, X3, r3, r1):
            X = X.cpu().numpy()
            for c in range(B.shape[0]):
                assert rk[c]["converged"] and rk[c]["relres_true"] <= tol, (kind, side, c, rk[c])
                assert _relres(A, X[c], B[c]) <= tol * 1.0001
                if rk0[c]["iterations"] > 25:
                    assert rk[c]["iterations"] < rk0[c]["iterations"], (rk[c]["iterations"], rk0[c]["iterations"])
