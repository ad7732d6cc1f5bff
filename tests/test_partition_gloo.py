"""The partitioned single forest's host side on two gloo ranks (CPU, 127.0.0.1).

Each rank computes its partition plan of the same adaptive forest with the
package's planner (no device involved) and the ranks check, over gloo, that the
plans agree: the same owner of every patch, every list one rank sends is the list
its peer expects, the substep weights are balanced.  The transport the solver calls
back into (forestclaw_b200.partition.TorchComm) moves packed halo buffers and
reduces arrays between the ranks through the same C-callback path the library
uses, here on host buffers."""
import ctypes
import datetime
import socket

import numpy as np


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import pyoracle as po
        from forestclaw_b200 import partition as pt
        from tests.cases import DAM, make
        oc, gc = make(DAM, mx=16, my=16, minlevel=2, maxlevel=5, subcycle=1, time_sync=1)
        o = po.OracleSim(oc)
        o.initialize()
        info = o.patch_info()
        p = pt.plan(gc, info[:, 0], info[:, 2], info[:, 3], rank, world)
        mine = torch.from_numpy(np.concatenate([p["owner"].astype(np.int64), p["nsend"].astype(np.int64),
                                                p["nrecv"].astype(np.int64), p["send_sum"].astype(np.int64),
                                                p["recv_sum"].astype(np.int64)]))
        allp = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(allp, mine)
        n = len(info)
        ok_plan = True
        for r in range(world):
            a = allp[r].numpy()
            ok_plan &= bool((a[:n] == allp[0].numpy()[:n]).all())
            for q in range(world):
                b = allp[q].numpy()
                ok_plan &= bool(a[n + q] == b[n + world + r])                    # counts r -> q
                ok_plan &= bool(a[n + 2 * world + q] == b[n + 3 * world + r])    # the same patches
        owner = allp[0].numpy()[:n]
        w = 2.0 ** (info[:, 0] - info[:, 0].min())
        loads = [float(w[owner == r].sum()) for r in range(world)]
        comm = pt.TorchComm(device=None)
        peer = 1 - rank
        send = np.arange(48, dtype=np.float64) + 1000.0 * rank
        recv = np.zeros(48)
        peers = (ctypes.c_int * 1)(peer)
        sp = (ctypes.c_void_p * 1)(send.ctypes.data)
        rp = (ctypes.c_void_p * 1)(recv.ctypes.data)
        sb = (ctypes.c_size_t * 1)(send.nbytes)
        rb = (ctypes.c_size_t * 1)(recv.nbytes)
        rc_x = comm.c.exchange(None, 1, peers, sp, sb, rp, rb)
        red = np.array([1.5 + rank, -2.0 * rank, 3.0])
        rc_m = comm.c.allreduce_max(None, red.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 3)
        tot = np.array([0.25 * (rank + 1), 1.0])
        rc_s = comm.c.allreduce_sum(None, tot.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 2)
        out.put((rank, ok_plan, loads, rc_x, recv.tolist(), rc_m, red.tolist(), rc_s, tot.tolist(), comm.failures))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_partition_plans_and_transport_on_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=240) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    for rank, ok_plan, loads, rc_x, recv, rc_m, red, rc_s, tot, failures in res:
        assert ok_plan and not failures
        assert abs(loads[0] - loads[1]) <= max(loads) * 0.05
        assert rc_x == 0 and recv == list(np.arange(48, dtype=np.float64) + 1000.0 * (1 - rank))
        assert rc_m == 0 and red == [2.5, 0.0, 3.0]
        assert rc_s == 0 and tot == [0.75, 2.0]
