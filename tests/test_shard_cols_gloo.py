"""The column-sharded build's host side on the CPU.

lgh_cols_range must tile the columns of a block contiguously in rank
order, in groups of four (so every rank's sub-block stays 16-byte aligned
for the vector kernels).  The torch.distributed communicator
(lgh_b200.dist.TorchComm) must gather equal-sized buffers in rank order:
two gloo ranks run its all-gather callback on CPU tensors exactly as the
library would call it, and reject an exchange outside its buffers.  No GPU
is touched."""

import os
import socket
from datetime import timedelta

import pytest

import lgh_b200 as L

WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("w,size", [(220, 2), (220, 8), (13, 4), (4, 3),
                                    (400, 3), (1, 1)])
def test_cols_range_tiles_the_block(w, size):
    cuts = [L.cols_range(w, r, size) for r in range(size)]
    assert cuts[0][0] == 0 and cuts[-1][1] == w
    for (a0, a1), (b0, b1) in zip(cuts, cuts[1:]):
        assert a1 == b0 and a0 <= a1
    for c0, c1 in cuts:
        assert c0 % 4 == 0
    widths = [b - a for a, b in cuts]
    assert max(widths) - min(widths) <= 4
    need = L.load().lgh_cols_exchange_bytes(1000, w, size)
    assert need >= 1000 * 8 * max(widths)


def _worker(rank, port, errq):
    try:
        import sys
        import torch
        import torch.distributed as dist
        sys.path.insert(0, os.path.dirname(os.path.dirname(
            os.path.abspath(__file__))))
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=WORLD,
                                timeout=timedelta(seconds=60))
        from lgh_b200.dist import torch_comm
        tc = torch_comm(n=100, max_cols=20, device="cpu")
        assert tc.comm.rank == rank and tc.comm.size == WORLD
        length = 100 * 8 * 7
        tc.send[:length] = (rank + 1) * 3
        rc = tc._allgather(tc.send.data_ptr(), tc.recv.data_ptr(), length, None)
        assert rc == 0, tc.error
        for r in range(WORLD):
            blk = tc.recv[r * length:(r + 1) * length]
            assert int(blk.min()) == int(blk.max()) == (r + 1) * 3
        # a buffer the communicator does not own is refused, not gathered
        other = torch.zeros(16, dtype=torch.uint8)
        assert tc._allgather(other.data_ptr(), tc.recv.data_ptr(), 8, None) == 1
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:                 # pragma: no cover - reported
        import traceback
        errq.put("rank %d: %s\n%s" % (rank, e, traceback.format_exc()))
        raise


def test_torch_comm_allgather_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, errq))
             for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
    errs = []
    while not errq.empty():
        errs.append(errq.get())
    assert not errs, errs
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
