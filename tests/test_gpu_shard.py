"""Device side of the row-sharded path on one GPU: two ranks' plans in one
process (no rank waits on another), the halo rows moved with
lgh_shard_pack / lgh_shard_unpack through device buffers, and the
extended blocks checked against the rows they stand for; the sharded
sketch rows (lgh_sketch_rows) against the same rows of the global sketch,
bit for bit."""

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

pytestmark = pytest.mark.gpu


def test_device_halo_pack_unpack(cuda_device):
    import torch
    cfg = P.grid_problem("c1")
    B, N = cfg["B"], cfg["N"]
    world, w = 2, 6
    shards = [L.Shard(B, world, r) for r in range(world)]
    ghosts = [s.ghosts() for s in shards]
    for r, s in enumerate(shards):
        for peer in range(world):
            if peer != r:
                g, c = ghosts[peer]
                first = int(np.sum(c[:r]))
                s.set_sends(peer, g[first:first + c[r]])
    X = np.random.default_rng(5).standard_normal((N, w))
    Lb = L.load()
    Xd = [torch.from_numpy(np.ascontiguousarray(X[s.row0:s.row1])).cuda()
          for s in shards]
    Xext = [torch.zeros((s.nloc + len(ghosts[r][0]), w), dtype=torch.float64,
                        device="cuda") for r, s in enumerate(shards)]
    for r, s in enumerate(shards):
        Xext[r][:s.nloc] = Xd[r]
    for src, s in enumerate(shards):
        for dst in range(world):
            if dst == src:
                continue
            cnt = len(s.sends(dst))
            buf = torch.empty((cnt, w), dtype=torch.float64, device="cuda")
            L._chk(Lb.lgh_shard_pack(s.h, dst, w, Xd[src].data_ptr(), w,
                                     buf.data_ptr()), "pack")
            L._chk(Lb.lgh_shard_unpack(shards[dst].h, src, w, buf.data_ptr(),
                                       Xext[dst].data_ptr(), w), "unpack")
    torch.cuda.synchronize()
    for r, s in enumerate(shards):
        ext = Xext[r].cpu().numpy()
        rows = np.concatenate([np.arange(s.row0, s.row1), ghosts[r][0]])
        assert np.array_equal(ext, X[rows])


def test_sketch_rows_partition_independent(cuda_device):
    import torch
    N, k, seed = 1000, 24, 271828
    full = L.test_sketch(seed, N, 0, k)
    for i0, n in ((0, 333), (333, 334), (667, 333), (999, 1)):
        ld = 28
        Y = torch.empty((n, ld), dtype=torch.float64, device="cuda")
        L._chk(L.load().lgh_sketch_rows(seed, i0, n, 0, k, Y.data_ptr(), ld),
               "lgh_sketch_rows")
        y = Y.cpu().numpy()
        assert np.array_equal(y[:, :k], full[i0:i0 + n])
        assert not y[:, k:].any()
