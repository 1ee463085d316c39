"""CPU tests: the batch launch's team sizes and list schedule
(mf_batch_schedule, the host code the batch uses).

The launch is cooperative (every block resident), and team members wait for
each other at bounded barriers; the schedule must therefore never make two
teams wait on each other: every block's list follows one global order of the
team items.  These tests check that order and the sizing rules on the list of the
512-system batch (seed 3) and on random cost sets."""
import math

import numpy as np
import pytest


def _item_costs(specs, cap=8):
    cost, tilem = [], []
    for kind, side, nr, n, nnz in specs:
        for c0 in range(0, nr, cap):
            g = min(cap, nr - c0)
            w = 8 if g >= 5 else 4 if g >= 3 else 2 if g == 2 else 1
            cost.append((n + nnz / 64.0) * (1.0 + 0.35 * (w - 1)) * n ** 0.4)
            tilem.append((n + 15) // 16)
    return cost, tilem


def _check(mf, cost, tilem, grid):
    team, lists, queue = mf.batch_schedule(cost, tilem, grid)
    n = len(cost)
    fair = sum(cost) / grid
    # sizing: round(4 cost / fair), capped by the launch and by one block per 64 tile-rows
    for t in range(n):
        want = math.floor(4.0 * cost[t] / fair + 0.5) if grid > 1 and fair > 0 else 1
        k = max(1, min(want, min(grid, max(1, tilem[t] // 64))))
        assert team[t] == (k if k >= 2 else 1), (t, team[t], k)
    # every team item: exactly team[t] entries, ranks 0..k-1, on distinct blocks
    where = {}
    for b, lst in enumerate(lists):
        for pos, (t, r) in enumerate(lst):
            where.setdefault(t, []).append((b, r, pos))
    for t in range(n):
        if team[t] > 1:
            e = where[t]
            assert sorted(r for _, r, _ in e) == list(range(team[t]))
            assert len({b for b, _, _ in e}) == team[t]
        else:
            assert t not in where
    # no two teams wait on each other: one global order of team items that every list follows
    order = {}
    for lst in lists:
        for a, b in zip(lst, lst[1:]):
            order.setdefault(a[0], set()).add(b[0])
    seen = {}

    def acyclic(u):
        seen[u] = 1
        for v in order.get(u, ()):
            if seen.get(v) == 1 or (v not in seen and not acyclic(v)):
                return False
        seen[u] = 2
        return True
    assert all(acyclic(u) for u in list(order) if u not in seen)
    # queue: the single-block items, largest cost first (stable)
    single = [t for t in range(n) if team[t] == 1]
    assert queue == sorted(single, key=lambda t: (-cost[t], t))
    return team, lists, queue


def test_schedule_on_the_512_system_batch(mf):
    from millefeuille import matrices as M
    cost, tilem = _item_costs(M.batch_specs(512, seed=3))
    for grid in (148, 296):
        team, lists, queue = _check(mf, cost, tilem, grid)
        assert sum(k > 1 for k in team) > 50 and len(queue) > 100
        # list scheduling keeps the team part within about one fair share of its load per block
        load = np.zeros(grid)
        for t, k in enumerate(team):
            if k > 1:
                for b, lst in enumerate(lists):
                    if any(e[0] == t for e in lst):
                        load[b] += cost[t] / k
        assert load.max() <= 1.5 * sum(cost) / grid


@pytest.mark.parametrize("seed", range(6))
def test_schedule_random(mf, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 400))
    cost = list(np.exp(rng.normal(0, 2.0, n)))
    tilem = [int(v) for v in rng.integers(1, 20000, n)]
    grid = int(rng.choice([1, 2, 7, 148, 296]))
    _check(mf, cost, tilem, grid)


def test_schedule_rejects_bad_input(mf):
    with pytest.raises(mf.MFError):
        mf.batch_schedule([1.0], [10], 0)
    with pytest.raises(mf.MFError):
        mf.batch_schedule([float("nan")], [10], 4)
