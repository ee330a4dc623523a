"""The row-sharded (N > 1) path on the CPU: two gloo ranks.

Each rank builds the shard plan of its row slab of the config-1 B operator
(lgh_shard_create: owned rows, ghost rows by owner, local column indices),
the ranks exchange their ghost requests (all-gather of the per-owner lists,
the all-to-all of the reference's VecScatter set-up), register them as
sends, exchange the halo rows of a seeded block, and multiply their local
CSR on the extended block [owned; ghosts].  The result must equal the same
rows of the global product; the all-reduced local Gram must equal the
global Gram; the benchmark's timing reduction must return the slowest
rank's time.  No GPU is touched (the plan is host code)."""

import os
import socket
from datetime import timedelta

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _csr_mult(rowptr, colidx, vals, X):
    Y = np.zeros((len(rowptr) - 1, X.shape[1]))
    for i in range(len(rowptr) - 1):
        k0, k1 = rowptr[i], rowptr[i + 1]
        Y[i] = vals[k0:k1] @ X[colidx[k0:k1]]
    return Y


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
        cfg = P.grid_problem("c1")
        B, N = cfg["B"], cfg["N"]
        sh = L.Shard(B, WORLD, rank)
        r0, r1 = sh.row0, sh.row1
        ghosts, counts = sh.ghosts()
        assert counts[rank] == 0 and counts.sum() == len(ghosts)
        assert np.all(np.diff(ghosts) > 0)
        assert np.all((ghosts < r0) | (ghosts >= r1))
        # local numbering: owned c -> c - r0, ghosts -> nloc + position
        lc = sh.local_colidx()
        ext = np.concatenate([np.arange(r0, r1), ghosts])
        assert np.array_equal(ext[lc], sh.colidx)
        # ghost requests to their owners
        first = np.concatenate([[0], np.cumsum(counts)])
        req = [ghosts[first[o]:first[o + 1]] for o in range(WORLD)]
        allreq = [None] * WORLD
        dist.all_gather_object(allreq, req)
        for peer in range(WORLD):
            if peer != rank:
                sh.set_sends(peer, allreq[peer][rank])
                assert np.array_equal(sh.sends(peer) + r0,
                                      allreq[peer][rank])
        # halo exchange of a seeded block, then the local product
        w = 5
        X = np.random.default_rng(17).standard_normal((N, w))
        Xloc = X[r0:r1]
        out = [Xloc[sh.sends(p)] if p != rank else None for p in range(WORLD)]
        allout = [None] * WORLD
        dist.all_gather_object(allout, out)
        recv = [allout[p][rank] for p in range(WORLD) if p != rank]
        Xext = np.vstack([Xloc] + recv)
        Y = _csr_mult(sh.rowptr, lc, sh.vals, Xext)
        ref = _csr_mult(B["rowptr"], B["colidx"], B["vals"], X)[r0:r1]
        assert np.allclose(Y, ref, rtol=1e-13, atol=1e-30)
        # Gram: local product + all-reduce
        G = torch.from_numpy(Xloc.T @ Xloc)
        dist.all_reduce(G)
        assert np.allclose(G.numpy(), X.T @ X, rtol=1e-12)
        # the benchmark's timing reduction: the slowest rank's time
        import bench
        t = bench.max_over_ranks(1.0 + rank, WORLD, "cpu")
        assert t == float(WORLD)
        sh.close()
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:  # report to the parent
        errq.put("rank %d: %r" % (rank, e))
        raise


def test_shard_plan_and_halo_exchange_two_ranks():
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


@pytest.mark.parametrize("N,P", [(1, 1), (7, 3), (4096, 2), (10, 4),
                                 (1000003, 8)])
def test_shard_range_partition(N, P):
    cuts = [L.shard_range(N, P, r) for r in range(P)]
    assert cuts[0][0] == 0 and cuts[-1][1] == N
    for (a0, a1), (b0, b1) in zip(cuts, cuts[1:]):
        assert a1 == b0 and a0 <= a1
    sizes = [b - a for a, b in cuts]
    assert max(sizes) - min(sizes) <= 1


def test_shard_rejects_bad_columns():
    csr = dict(rowptr=np.array([0, 1, 2], np.int64),
               colidx=np.array([0, 5], np.int32))
    with pytest.raises(L.LghError) as e:
        L.Shard(csr, 1, 0)
    assert e.value.code == 63
