"""CPU tests: the split of a batch over GPUs (mf_batch_partition) and the
host-side gather of a sharded batch's reports, with world_size-2 gloo ranks.

The split has no reference counterpart; it is checked against a direct
restatement of greedy longest-processing-time over the documented cost, and
against Graham's bound (largest load <= mean load + largest cost)."""
import math
import os
import socket

import numpy as np
import pytest


def _cost(n, nnz, nrhs, cap=8):
    c = 0.0
    for c0 in range(0, nrhs, cap):
        g = min(cap, nrhs - c0)
        w = 8 if g >= 5 else 4 if g >= 3 else 2 if g == 2 else 1
        c += (max(n, 1) + nnz / 64.0) * (1.0 + 0.35 * (w - 1)) * max(n, 1) ** 0.4
    return c


def _lpt(costs, nparts):
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    load = [0.0] * nparts
    part = [0] * len(costs)
    for k in order:
        q = min(range(nparts), key=lambda j: (load[j], j))
        part[k] = q
        load[q] += costs[k]
    return part, load


@pytest.mark.parametrize("nparts,cap", [(1, 8), (2, 8), (3, 4), (8, 8), (8, 2)])
def test_partition_is_lpt_over_the_queue_cost(mf, nparts, cap):
    from millefeuille import matrices as M, shard
    specs = M.batch_specs(512, seed=3)
    n, nnz, nr = [s[3] for s in specs], [s[4] for s in specs], [s[2] for s in specs]
    part, load = shard.partition(n, nnz, nr, nparts, cap=cap)
    costs = [_cost(a, b, c, cap) for a, b, c in zip(n, nnz, nr)]
    part_ref, load_ref = _lpt(costs, nparts)
    assert part == part_ref
    np.testing.assert_allclose(load, load_ref, rtol=1e-12)
    assert sorted(k for q in range(nparts) for k in shard.owned(part, q)) == list(range(512))
    assert shard.lpt_bound_ok(part, costs, nparts)
    if nparts > 1:
        assert max(load) / (sum(load) / nparts) < 1.05          # 512 systems split evenly
    assert shard.partition(n, nnz, nr, nparts, cap=cap) == (part, load)   # deterministic


def test_partition_edges(mf):
    from millefeuille import shard
    part, load = shard.partition([100, 50], [500, 200], [1, 3], 4)
    assert sorted(part) == [0, 1] and load[2] == 0.0 and load[3] == 0.0    # more GPUs than systems
    assert shard.partition([], [], [], 3) == ([], [0.0, 0.0, 0.0])
    # equal costs: ties go to the lower system index and the lower part
    assert shard.partition([64] * 4, [320] * 4, [2] * 4, 2)[0] == [0, 1, 0, 1]
    with pytest.raises(mf.MFError):
        shard.partition([10], [50], [0], 2)           # a system without right-hand sides
    with pytest.raises(mf.MFError):
        shard.partition([10], [50], [1], 0)           # no parts
    with pytest.raises(mf.MFError):
        shard.partition([10], [50], [1], 2, cap=9)    # wider than a work item


def test_batch_specs_match_the_generator():
    from millefeuille import matrices as M
    kw = dict(side2d=(6, 30), side3d=(3, 9), rhs=(1, 16))
    specs = M.batch_specs(12, seed=5, **kw)
    full = M.batch_systems(12, seed=5, **kw)
    for (kind, side, nr, n, nnz), (k2, s2, A, B) in zip(specs, full):
        assert (kind, side, n, nnz, nr) == (k2, s2, A.n, A.nnz, B.shape[0])
    sub = M.batch_systems(12, seed=5, only=[9, 4], **kw)
    for (k, s, A, B), j in zip(sub, [9, 4]):
        assert np.array_equal(A.val, full[j][2].val) and np.array_equal(B, full[j][3])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import json
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "..", "mille-feuille_b200"))
    from millefeuille import matrices as M, shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        specs = M.batch_specs(64, seed=3, side2d=(6, 30), side3d=(3, 9), rhs=(1, 16))
        part, _ = shard.partition([s[3] for s in specs], [s[4] for s in specs], [s[2] for s in specs], world)
        parts = [None] * world
        dist.all_gather_object(parts, part)
        own = shard.owned(part, rank)
        # stand-in for this rank's mf_batch solve: one report per column, tagged
        reps = [[{"system": k, "column": c, "rank": rank} for c in range(specs[k][2])] for k in own]
        full = shard.gather_reports(own, reps, len(specs))
        slowest = shard.max_over_ranks(1.5 + rank)
        res = {"same_split": all(p == part for p in parts), "slowest": slowest, "n_own": len(own)}
        if rank == 0:
            res["systems"] = [[r["system"] for r in rk] for rk in full]
            res["columns"] = [len(rk) for rk in full]
            res["owner_ok"] = all(r["rank"] == part[k] for k, rk in enumerate(full) for r in rk)
        else:
            res["full_is_none"] = full is None
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def test_sharded_reports_gather_gloo(tmp_path):
    """Two gloo ranks: identical split without communication, every system's
    reports gathered on rank 0 exactly once, in system order; the batch time
    is the slowest rank's."""
    import json
    import torch.multiprocessing as tmp
    from millefeuille import matrices as M
    world = 2
    tmp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                        start_method="spawn")
    r = [json.load(open(tmp_path / f"rank{q}.json")) for q in range(world)]
    specs = M.batch_specs(64, seed=3, side2d=(6, 30), side3d=(3, 9), rhs=(1, 16))
    assert r[0]["same_split"] and r[1]["same_split"]
    assert r[0]["n_own"] + r[1]["n_own"] == 64 and min(r[0]["n_own"], r[1]["n_own"]) > 0
    assert r[0]["systems"] == [[k] * s[2] for k, s in enumerate(specs)]
    assert r[0]["columns"] == [s[2] for s in specs] and r[0]["owner_ok"]
    assert r[1]["full_is_none"]
    assert r[0]["slowest"] == r[1]["slowest"] == 2.5
