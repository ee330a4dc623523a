"""torch.distributed communicators for the sharded builds.

Column-sharded build (TorchComm):

lgh_glr_compute_cols (one rank per GPU) needs an all-gather of equal-sized
device buffers after each F-apply.  `torch_comm` makes the lgh_comm_t that
does it over a torch.distributed process group: the exchange buffers are
torch uint8 tensors on the rank's device (sized by lgh_cols_exchange_bytes
for the widest block the object will apply F to), and the callback runs
all_gather_into_tensor on them (NCCL over NVLink on a GPU node; on gloo a
list all-gather into views of the receive buffer).  The library calls the
callback from the thread that called it, in the same order on every rank.
"""

import ctypes

import numpy as np

from . import (ALLGATHER_FN, ROWS_ALLREDUCE_FN, ROWS_ALLTOALLV_FN, Comm,
               RowsComm, load)


class TorchComm:
    """Owns the exchange tensors and the callback for one rank."""

    def __init__(self, n, max_cols, device, group=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        nbytes = int(load().lgh_cols_exchange_bytes(n, max_cols, self.size))
        self.send = torch.empty(nbytes, dtype=torch.uint8, device=device)
        self.recv = torch.empty(nbytes * self.size, dtype=torch.uint8,
                                device=device)
        self.backend = dist.get_backend(group)
        self.calls = 0
        self.error = None
        self._cb = ALLGATHER_FN(self._allgather)
        self.comm = Comm(rank=self.rank, size=self.size,
                         send=self.send.data_ptr(), recv=self.recv.data_ptr(),
                         bytes=nbytes, allgather=self._cb, ctx=None)

    def _allgather(self, sp, rp, length, ctx):
        try:
            if sp != self.send.data_ptr() or rp != self.recv.data_ptr() \
                    or length > self.send.numel():
                raise ValueError("exchange outside the communicator's buffers")
            inp = self.send[:length]
            out = self.recv[:length * self.size]
            if self.backend == "nccl":
                self.dist.all_gather_into_tensor(out, inp, group=self.group)
            else:
                views = [out[r * length:(r + 1) * length]
                         for r in range(self.size)]
                self.dist.all_gather(views, inp, group=self.group)
            self.calls += 1
            return 0
        except Exception as e:       # reported to the library as a failure
            self.error = repr(e)
            return 1


def torch_comm(n, max_cols, device, group=None):
    return TorchComm(n, max_cols, device, group)


class _DevBuf:
    """A raw device range seen by torch.as_tensor (CUDA array interface)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {
            "shape": (int(count),), "typestr": typestr,
            "data": (int(ptr), False), "version": 3, "strides": None}


def _wrap(ptr, count, dtype, device):
    """A tensor over count elements at ptr (device memory, or host memory
    for a CPU device), without a copy."""
    import torch
    if count == 0:
        return torch.empty(0, dtype=dtype, device=device)
    if torch.device(device).type == "cuda":
        ts = {torch.float64: "<f8", torch.uint8: "|u1"}[dtype]
        return torch.as_tensor(_DevBuf(ptr, count, ts), device=device)
    ct = {torch.float64: ctypes.c_double, torch.uint8: ctypes.c_uint8}[dtype]
    arr = np.ctypeslib.as_array((ct * int(count)).from_address(int(ptr)))
    return torch.from_numpy(arr)


class TorchRowsComm:
    """The lgh_rows_comm_t of one rank for the build over row slabs.

    allreduce: dist.all_reduce (SUM) in place on the library's FP64 buffer;
    every rank receives the same sum.  alltoallv: all_to_all_single with
    byte split sizes on NCCL; on gloo (which has no all-to-all) one isend /
    irecv pair per peer.  Each callback completes the collective before it
    returns (the library reads the results next)."""

    def __init__(self, device, group=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.device = torch.device(device)
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.backend = dist.get_backend(group)
        self.calls = {"allreduce": 0, "alltoallv": 0}
        self.error = None
        self._ar = ROWS_ALLREDUCE_FN(self._allreduce)
        self._a2a = ROWS_ALLTOALLV_FN(self._alltoallv)
        self.comm = RowsComm(rank=self.rank, size=self.size,
                             allreduce=self._ar, alltoallv=self._a2a,
                             ctx=None)

    def _sync(self):
        if self.device.type == "cuda":
            self.torch.cuda.synchronize(self.device)

    def _allreduce(self, buf, count, ctx):
        try:
            t = _wrap(buf, count, self.torch.float64, self.device)
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM,
                                 group=self.group)
            self._sync()
            self.calls["allreduce"] += 1
            return 0
        except Exception as e:       # reported to the library as a failure
            self.error = repr(e)
            return 1

    def _alltoallv(self, send, sbytes, recv, rbytes, ctx):
        try:
            torch, dist = self.torch, self.dist
            sb = [int(sbytes[p]) for p in range(self.size)]
            rb = [int(rbytes[p]) for p in range(self.size)]
            st = _wrap(send, sum(sb), torch.uint8, self.device)
            rt = _wrap(recv, sum(rb), torch.uint8, self.device)
            if self.backend == "nccl":
                dist.all_to_all_single(rt, st, output_split_sizes=rb,
                                       input_split_sizes=sb, group=self.group)
            else:
                so = np.concatenate([[0], np.cumsum(sb)]).astype(int)
                ro = np.concatenate([[0], np.cumsum(rb)]).astype(int)
                reqs = []
                for p in range(self.size):
                    if p == self.rank:
                        continue
                    peer = dist.get_global_rank(self.group, p) \
                        if self.group is not None else p
                    if rb[p]:
                        reqs.append(dist.irecv(rt[ro[p]:ro[p + 1]], peer,
                                               group=self.group))
                    if sb[p]:
                        reqs.append(dist.isend(st[so[p]:so[p + 1]], peer,
                                               group=self.group))
                for r in reqs:
                    r.wait()
            self._sync()
            self.calls["alltoallv"] += 1
            return 0
        except Exception as e:       # reported to the library as a failure
            self.error = repr(e)
            return 1


def torch_rows_comm(device, group=None):
    return TorchRowsComm(device, group)


__all__ = ["TorchComm", "torch_comm", "TorchRowsComm", "torch_rows_comm"]
