"""A torch.distributed communicator for the column-sharded build.

lgh_glr_compute_cols (one rank per GPU) needs an all-gather of equal-sized
device buffers after each F-apply.  `torch_comm` makes the lgh_comm_t that
does it over a torch.distributed process group: the exchange buffers are
torch uint8 tensors on the rank's device (sized by lgh_cols_exchange_bytes
for the widest block the object will apply F to), and the callback runs
all_gather_into_tensor on them (NCCL over NVLink on a GPU node; on gloo a
list all-gather into views of the receive buffer).  The library calls the
callback from the thread that called it, in the same order on every rank.
"""

from . import ALLGATHER_FN, Comm, load


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


__all__ = ["TorchComm", "torch_comm"]
