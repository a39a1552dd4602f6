"""Multi-rank density scan on CPU: the partition and the gather, two gloo ranks.

The solves are replaced by a deterministic stand-in (no GPU): the test covers
the host logic that shards a scan across processes and reassembles the results."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from jax_hf_b200.scan import partition_solves, solve_cost, solve_scan


def test_partition_is_balanced_and_complete():
    costs = [solve_cost(nk, nk, nb) for nk, nb in [(120, 8), (36, 4), (96, 6), (48, 8), (72, 4), (120, 4), (36, 8)]]
    parts = partition_solves(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / 3 + max(costs)  # LPT bound
    assert partition_solves(costs, 3) == parts  # deterministic
    with pytest.raises(ValueError):
        partition_solves(costs, 0)


def test_single_process_scan_keeps_order():
    shapes = [(12, 12, 4), (24, 24, 8), (16, 16, 6)]
    out = solve_scan(shapes, lambda idx: [dict(i=i) for i in idx])
    assert [o["i"] for o in out] == [0, 1, 2]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, shapes, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ran = []

        def run_local(idx):
            ran.extend(idx)
            return [dict(i=i, value=float(i) ** 2 + 0.5, rank=rank) for i in idx]

        out = solve_scan(shapes, run_local)
        q.put((rank, sorted(ran), [(o["i"], o["value"]) for o in out]))
    finally:
        dist.destroy_process_group()


def test_two_rank_scan_shards_and_gathers():
    shapes = [(36, 36, 4), (120, 120, 8), (48, 48, 6), (96, 96, 8), (72, 72, 4), (120, 120, 4), (36, 36, 8)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, shapes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    ran0, ran1 = res[0][1], res[1][1]
    assert sorted(ran0 + ran1) == list(range(len(shapes))) and not set(ran0) & set(ran1)
    expect = [(i, float(i) ** 2 + 0.5) for i in range(len(shapes))]
    assert res[0][2] == expect and res[1][2] == expect
