"""Ensemble partitioning over ranks (no GPU): the longest-processing-time partition,
memory grouping, and a world_size-2 gloo run whose gathered results equal a
single-process run member for member (the oracle stands in for the device)."""
import socket

import numpy as np
import pytest

from imau_ice_b200 import diva, ensemble
import dist_worker


def test_partition_assigns_every_member_once_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.integers(1, 1000, 37).astype(float))
    for nr in (1, 2, 3, 8):
        parts = ensemble.partition(costs, nr)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[k] for k in p) for p in parts]
        # LPT bound: the largest load exceeds the mean by less than the largest item
        assert max(loads) <= sum(costs) / nr + max(costs)
    assert ensemble.partition(costs, 4) == ensemble.partition(costs, 4)    # deterministic


def test_partition_known_answer():
    # decreasing order 7 5 4 3 1 onto 2 ranks: r0 7, r1 5, r1 4 (9), r0 3 (10), r1 1 (10)
    assert ensemble.partition([3, 7, 1, 5, 4], 2) == [[0, 1], [2, 3, 4]]


def test_groups_respect_the_memory_budget():
    g_small, g_big = diva.Grid(129, 17, 5e3), diva.Grid(1501, 1501, 4e3)
    members = [("channel-0", g_small, {}, {}), ("sheet-1", g_big, {}, {}), ("channel-2", g_small, {}, {})]
    per = [ensemble.BYTES_PER_COLUMN * g.nx * g.ny for _, g, _, _ in members]
    gr = ensemble.groups(members, [0, 1, 2], budget_bytes=per[1] * 0.5)
    assert gr == [[0], [1], [2]]                     # the big one alone, over budget by itself
    assert ensemble.groups(members, [0, 2], budget_bytes=1e12) == [[0, 2]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gloo_equal_one_process(oracle):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=dist_worker.ensemble_rank,
                         args=(r, 2, port, q, dist_worker.small_channel_members)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    one, _ = ensemble.solve_ensemble(dist_worker.small_channel_members(), oracle, 0, 1)
    parts = got[0][2]
    assert sorted(parts[0] + parts[1]) == [0, 1, 2, 3] and parts[0] and parts[1]
    for rank, res, _ in got:
        assert sorted(res) == [0, 1, 2, 3]            # every rank holds every member after the gather
        for k, (its, u, v) in res.items():
            assert its == one[k]["report"]["picard_iterations"]
            assert np.array_equal(u, one[k]["u_vav_cx"]) and np.array_equal(v, one[k]["v_vav_cy"])
