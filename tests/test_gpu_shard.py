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


def test_cols_sharded_build_two_ranks_on_one_device(cuda_device):
    """The column-sharded build with two ranks run as threads on one GPU
    (the in-process communicator: a host barrier and device copies, no
    kernel waits on another rank).  Each rank owns half of the sketch
    columns; after the build both ranks hold the same object, equal to
    the one-device build on the same inputs (same hashed sketch), and the
    sharded extension equals the one-device extension."""
    import threading
    cfg = P.grid_problem("c1")
    o = L.glr_opts(ell=60, seed=0, trunc_rel=1e-3, check=1)
    one = {}

    def objs():
        B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
        pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-12))
        return B, Z, pr

    keep1 = objs()
    g1 = L.Glr(keep1[0], keep1[2], o)
    comms = L.local_comms(2)
    res, errs = [None, None], []

    def rank(r):
        try:
            keep = objs()
            g = L.Glr(keep[0], keep[2], o, comm=comms[r])
            rep0 = dict(g.report)
            g.extend(20)
            res[r] = (g.eigs(), g.U(), rep0, keep, g)
        except Exception as e:             # reported below
            errs.append(repr(e))

    th = [threading.Thread(target=rank, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    (l0, U0, rep0, _, _), (l1, U1, rep1, _, _) = res
    assert np.array_equal(l0, l1) and np.array_equal(U0, U1)
    lo = g1.eigs()
    assert len(lo) == rep0["kept"]
    assert abs(rep0["resid_max"] - g1.report["resid_max"]) \
        < 1e-3 * g1.report["resid_max"]
    g1.extend(20)
    l1x = g1.eigs()
    assert len(l1x) == len(l0)
    assert np.max(np.abs(l0 - l1x) / l1x) < 1e-10
    L.free_local_comms(comms)
