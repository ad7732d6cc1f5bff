"""One forest partitioned over ranks: the communicator callbacks of
fc2d_b200_set_partition over a torch.distributed process group.

The library calls back between the launches of an advance (its stream idle):
``exchange`` sends each peer its packed halo segment and receives the peer's
(device buffers; NCCL moves them device to device, gloo through host staging),
``allreduce_max`` / ``allreduce_sum`` reduce small host arrays (CFL number and
status, regrid tags, mass partials).  Every rank makes the same calls in the same
order.  The reference's counterparts are fclaw2d_exchange_ghost_patches_begin/end
(src/fclaw2d_exchange.c:308-413) and fclaw2d_domain_global_maximum / _sum.
"""
from __future__ import annotations

import ctypes

import numpy as np

EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                               ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t))
REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int)


class Comm(ctypes.Structure):
    """fc2d_b200_comm_t."""
    _fields_ = [("rank", ctypes.c_int), ("size", ctypes.c_int), ("user", ctypes.c_void_p),
                ("exchange", EXCHANGE_FN), ("allreduce_max", REDUCE_FN), ("allreduce_sum", REDUCE_FN)]


class _DeviceBuffer:
    """A raw device range seen as a float64 array (CUDA array interface)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes // 8,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


class TorchComm:
    """Callbacks over the default torch.distributed group.  device: the CUDA device
    of the solver (its buffers are device memory), or None when the buffers the
    library hands over are host memory (tests of the transport alone)."""

    def __init__(self, device: int | None = 0):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.device = device
        self.nccl = dist.get_backend() == "nccl"
        self._keep = (EXCHANGE_FN(self._exchange), REDUCE_FN(self._max), REDUCE_FN(self._sum))
        self.c = Comm(self.rank, self.size, None, *self._keep)
        self.failures = []

    def exchange_arrays(self, peers, sends, recvs):
        """Send sends[k] to peers[k] and receive recvs[k] from it (torch tensors)."""
        import torch
        staged = self.device is not None and not self.nccl          # gloo: through host memory
        hs = [x.cpu() for x in sends] if staged else list(sends)
        hr = [torch.empty_like(x, device="cpu") for x in recvs] if staged else list(recvs)
        ops = []
        for p, snd, rcv in zip(peers, hs, hr):
            if snd.numel():
                ops.append(self.dist.P2POp(self.dist.isend, snd, p))
            if rcv.numel():
                ops.append(self.dist.P2POp(self.dist.irecv, rcv, p))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        if staged:
            for r, h in zip(recvs, hr):
                r.copy_(h)
        if self.device is not None:
            torch.cuda.synchronize(self.device)

    def _view(self, ptr, nbytes):
        import torch
        if self.device is None:
            buf = (ctypes.c_double * (nbytes // 8)).from_address(ptr)
            return torch.from_numpy(np.ctypeslib.as_array(buf))
        return torch.as_tensor(_DeviceBuffer(ptr, nbytes), device=f"cuda:{self.device}")

    def _exchange(self, user, npeers, peers, send, send_bytes, recv, recv_bytes):
        try:
            pr = [peers[k] for k in range(npeers)]
            snd = [self._view(send[k], send_bytes[k]) for k in range(npeers)]
            rcv = [self._view(recv[k], recv_bytes[k]) for k in range(npeers)]
            self.exchange_arrays(pr, snd, rcv)
            return 0
        except Exception as e:                                 # noqa: BLE001 -- reported by the return code
            self.failures.append(repr(e))
            return 1

    def _reduce(self, v, n, op):
        import torch
        try:
            a = np.ctypeslib.as_array(v, shape=(n,))
            t = torch.from_numpy(a.copy())
            if self.nccl:
                t = t.to(f"cuda:{self.device}")
            self.dist.all_reduce(t, op=op)
            a[:] = t.cpu().numpy()
            return 0
        except Exception as e:                                 # noqa: BLE001
            self.failures.append(repr(e))
            return 1

    def _max(self, user, v, n):
        return self._reduce(v, n, self.dist.ReduceOp.MAX)

    def _sum(self, user, v, n):
        return self._reduce(v, n, self.dist.ReduceOp.SUM)


def partition(solver, comm: TorchComm | None) -> None:
    """Partition solver's forest over comm's ranks (None: back to one rank)."""
    rc = solver.lib.fc2d_b200_set_partition(solver.h, ctypes.byref(comm.c) if comm is not None else None)
    solver._check("fc2d_b200_set_partition", rc)
    solver._comm = comm                                        # the callbacks live as long as the solver


def plan(opts, level, gx, gy, rank: int, size: int) -> dict:
    """The partition plan of `rank` for a forest (host only, no device)."""
    import forestclaw_b200 as fb
    lib = fb.load_library()
    n = len(level)
    arrs = [np.ascontiguousarray(a, np.int32) for a in (level, gx, gy)]
    owner = np.zeros(n, np.int32)
    ns, nr = np.zeros(size, np.int32), np.zeros(size, np.int32)
    ss, rs = np.zeros(size, np.uint64), np.zeros(size, np.uint64)
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))  # noqa: E731
    up = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong))  # noqa: E731
    c = opts.to_c()
    rc = lib.fc2d_b200_partition_plan(ctypes.byref(c), n, *[ip(a) for a in arrs], rank, size, ip(owner), ip(ns),
                                      ip(nr), up(ss), up(rs))
    if rc != 0:
        raise fb.B200Error("fc2d_b200_partition_plan", rc, (lib.fc2d_b200_last_error() or b"").decode())
    return {"owner": owner, "nsend": ns, "nrecv": nr, "send_sum": ss, "recv_sum": rs}
