"""Multi-rank plumbing on the CPU: two gloo ranks (127.0.0.1) exercise what a
multi-GPU bench run does across ranks -- the device time is the maximum over
ranks, the work the sum, and batch ranks draw disjoint instance seeds -- with
the same collectives in the same order on every rank."""
import datetime
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from forestclaw_b200 import problems, ranks
        r, w = ranks.rank_world()
        agg = ranks.aggregate(10.0 + rank, 100.0 * (rank + 1), "cpu")
        base = ranks.instance_seed_base(rank, 64)
        insts, _ = problems.tsunami_instances(64, base)
        out.put((rank, r, w, agg, base, [tuple(i["pdata"]) for i in insts]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_and_shard():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=180) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    (r0, rr0, w0, agg0, b0, i0), (r1, rr1, w1, agg1, b1, i1) = res
    assert (rr0, w0, rr1, w1) == (0, 2, 1, 2)
    # max of 10 and 11 ms, sum of 100 and 200 cell updates, identical on both ranks
    assert agg0 == agg1 == (11.0, 300.0, pytest.approx(300.0 / 11e-3))
    assert (b0, b1) == (0, 64)
    assert not set(i0) & set(i1)          # disjoint instances: 128 distinct forests in all


def test_single_process_is_identity():
    from forestclaw_b200 import ranks
    assert ranks.rank_world() == (0, 1)
    assert ranks.aggregate(5.0, 50.0) == (5.0, 50.0, 50.0 / 5e-3)
