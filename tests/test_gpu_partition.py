"""One forest partitioned over ranks (fc2d_b200_set_partition), bit for bit.

Two and three ranks run as separate processes on the one GPU of the machine, each
with its own solver; the halo exchange goes through host memory over gloo
(forestclaw_b200.partition.TorchComm), between the launches of each rank's advance,
so no kernel waits on another process.  Subcycled AMR radial dam with time sync and
regrids: the CFL numbers of every step, the forest, every patch's q (gathered with
fc2d_b200_sync_replicas), the registers and the mass must equal a single-rank run."""
import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KW = dict(mx=16, my=16, minlevel=2, maxlevel=5, subcycle=1, time_sync=1)
STEPS, REGRID = 6, 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(g, part=None):
    t, dt, cfls = 0.0, 0.004, []
    for n in range(STEPS):
        c = g.advance(t, dt)
        cfls.append(c)
        t += dt
        dt *= 0.9 / c
        if (n + 1) % REGRID == 0:
            g.regrid()
    if part:
        g.sync_replicas()
    return cfls, g.patch_info(), g.get_q(), g.get_registers(), g.mass()


def _worker(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import forestclaw_b200 as fb
        from forestclaw_b200 import partition as pt
        from tests.cases import DAM, make
        _, gc = make(DAM, **KW)
        g = fb.Solver(gc)
        comm = pt.TorchComm(device=0)
        pt.partition(g, comm)
        g.initialize()
        owners = g.partition_owner()
        res = _run(g, part=True)
        out.put((rank, res, [int((owners == r).sum()) for r in range(world)], comm.failures))
        g.close()
        dist.barrier()
    except Exception as e:                              # noqa: BLE001
        out.put((rank, None, repr(e), []))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_forest_bitwise_with_one_rank(world):
    import multiprocessing as mp
    import forestclaw_b200 as fb
    from tests.cases import DAM, make
    _, gc = make(DAM, **KW)
    g = fb.Solver(gc)
    g.initialize()
    ref = _run(g)
    g.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    env = dict(os.environ)
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = sorted((q.get(timeout=300) for _ in range(world)), key=lambda x: x[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    del env
    for rank, r, counts, failures in res:
        assert r is not None, counts
        assert not failures
        assert min(counts) > 0                       # every rank owns patches
        cfls, info, qq, regs, mass = r
        assert cfls == ref[0], (rank, cfls, ref[0])
        assert np.array_equal(info, ref[1])
        assert np.array_equal(qq, ref[2])
        assert np.array_equal(regs, ref[3])
        assert np.array_equal(mass, ref[4])
