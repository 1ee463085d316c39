"""Batched solves split across GPUs: one process per GPU (torch.distributed
ranks), each owning whole systems and solving them with its own mf_batch.

The split is mf_batch_partition (greedy longest-processing-time over the work
queue's cost estimate), computed identically on every rank from the systems'
sizes, so choosing the split needs no communication and the solves need no
collective.  The only exchange is the host-side gather of the per-system
reports (and of the timings) after the solves.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check


def partition(n, nnz, nrhs, nparts: int, cap: int = 8):
    """Part of every system (list of ints, one per system) and every part's
    total estimated cost (list of floats)."""
    L = _lib.load()
    ns = len(n)
    if not (len(nnz) == ns and len(nrhs) == ns):
        raise ValueError("n, nnz and nrhs must have one entry per system")
    a_n = (C.c_int * max(ns, 1))(*[int(v) for v in n])
    a_z = (C.c_longlong * max(ns, 1))(*[int(v) for v in nnz])
    a_r = (C.c_int * max(ns, 1))(*[int(v) for v in nrhs])
    part = (C.c_int * max(ns, 1))()
    load = (C.c_double * nparts)()
    check(L.mf_batch_partition(ns, a_n, a_z, a_r, int(cap), int(nparts), part, load), "mf_batch_partition")
    return [int(part[k]) for k in range(ns)], [float(load[q]) for q in range(nparts)]


def owned(part, rank: int):
    """Indices of the systems that `rank` owns, in system order."""
    return [k for k, q in enumerate(part) if q == rank]


def gather_reports(own, reports, nsys: int, group=None, dst: int = 0):
    """Host-side gather of every rank's per-system reports to rank `dst`.

    own: this rank's system indices; reports: its per-system report lists in
    the same order.  Returns the full list in system order on `dst` (every
    system exactly once, else ValueError), None on the other ranks.  Every rank
    of the group must call it."""
    import torch.distributed as dist
    if len(own) != len(reports):
        raise ValueError("one report list per owned system")
    mine = list(zip([int(k) for k in own], reports))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    bucket = [None] * world if rank == dst else None
    dist.gather_object(mine, bucket, dst=dst, group=group)
    if rank != dst:
        return None
    full = [None] * nsys
    for part in bucket:
        for k, r in part:
            if not 0 <= k < nsys or full[k] is not None:
                raise ValueError(f"system {k} reported twice or out of range")
            full[k] = r
    missing = [k for k, r in enumerate(full) if r is None]
    if missing:
        raise ValueError(f"systems without a report: {missing[:8]}")
    return full


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest of every rank's value (the batch time of a sharded solve is
    the slowest rank's)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def lpt_bound_ok(part, cost, nparts: int) -> bool:
    """Graham's bound for greedy LPT: the largest load is at most the mean load
    plus the largest single cost (used by the tests)."""
    ld = np.zeros(nparts)
    for k, q in enumerate(part):
        ld[q] += cost[k]
    return bool(ld.max() <= ld.sum() / nparts + max(cost, default=0.0) + 1e-9 * max(1.0, ld.sum()))
