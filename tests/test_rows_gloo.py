"""The row-slab build's communicator on the CPU.

lgh_b200.dist.TorchRowsComm is what a torch.distributed job hands the
library for a build over row slabs (lgh_mat_create_rows, and the build,
solves and products on the sharded objects).  Three gloo ranks call its
two callbacks through their C function pointers, as the library does:

  - allreduce: every rank's FP64 buffer becomes the elementwise sum, the
    same bits on every rank (the library takes its PCG decisions from
    these sums, so the ranks must agree exactly);
  - alltoallv: ragged byte counts per peer, packed in peer order on both
    sides (the halo exchange and the plan exchange), zero-length chunks
    included.

Also the host helper that cuts a rank's slab out of a CSR operator, and
lgh_shard_range's even split (the rows each rank must own).  No GPU is
touched."""

import ctypes
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

import lgh_b200 as L
from lgh_b200 import problems

WORLD = 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_rows_slab_cuts_the_operator():
    rng = np.random.default_rng(3)
    n = 37
    D = (rng.random((n, n)) < 0.2) * rng.standard_normal((n, n))
    D = D + D.T + np.eye(n)
    A = problems.dense_to_csr(D)
    rows = []
    for r in range(WORLD):
        a, b = L.shard_range(n, WORLD, r)
        sl = L.rows_slab(A, a, b)
        assert sl["rowptr"][0] == 0 and len(sl["rowptr"]) == b - a + 1
        for i in range(b - a):
            k0, k1 = sl["rowptr"][i], sl["rowptr"][i + 1]
            row = np.zeros(n)
            row[np.asarray(sl["colidx"][k0:k1])] = sl["vals"][k0:k1]
            rows.append(row)
    assert np.array_equal(np.array(rows), D)
    # the even split: contiguous, covering, sizes differ by at most one
    cuts = [L.shard_range(n, WORLD, r) for r in range(WORLD)]
    assert cuts[0][0] == 0 and cuts[-1][1] == n
    assert all(a1 == b0 for (_, a1), (b0, _) in zip(cuts, cuts[1:]))
    sizes = [b - a for a, b in cuts]
    assert max(sizes) - min(sizes) <= 1


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
        from lgh_b200.dist import torch_rows_comm
        tc = torch_rows_comm(device="cpu")
        c = tc.comm
        assert c.rank == rank and c.size == WORLD

        # all-reduce in place, through the C function pointer
        count = 37
        buf = np.arange(count, dtype=np.float64) * 0.1 + (rank + 1) / 3.0
        assert c.allreduce(buf.ctypes.data, count, None) == 0, tc.error
        want = sum(np.arange(count) * 0.1 + (r + 1) / 3.0
                   for r in range(WORLD))
        assert np.allclose(buf, want, rtol=0, atol=1e-13)
        everyone = [None] * WORLD
        dist.all_gather_object(everyone, buf.tobytes())
        assert all(e == everyone[0] for e in everyone)   # the same bits

        # ragged all-to-all: rank r sends (r + 1) * (p + 2) - 2 bytes to p
        # (none to itself), each byte = 16 r + p
        def nbytes(src, dst):
            return 0 if src == dst else (src + 1) * (dst + 2) - 2
        sb = [nbytes(rank, p) for p in range(WORLD)]
        rb = [nbytes(p, rank) for p in range(WORLD)]
        send = np.concatenate([np.full(sb[p], 16 * rank + p, np.uint8)
                               for p in range(WORLD)])
        recv = np.full(sum(rb), 255, np.uint8)
        SB = (ctypes.c_size_t * WORLD)(*sb)
        RB = (ctypes.c_size_t * WORLD)(*rb)
        assert c.alltoallv(send.ctypes.data, SB, recv.ctypes.data, RB,
                           None) == 0, tc.error
        off = 0
        for p in range(WORLD):
            chunk = recv[off:off + rb[p]]
            assert np.all(chunk == 16 * p + rank), (p, chunk[:4])
            off += rb[p]
        assert tc.calls == {"allreduce": 1, "alltoallv": 1}
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:                 # pragma: no cover - reported
        import traceback
        errq.put("rank %d: %s\n%s" % (rank, e, traceback.format_exc()))
        raise


def test_torch_rows_comm_three_gloo_ranks():
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
