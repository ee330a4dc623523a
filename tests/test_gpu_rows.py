"""The build over row slabs on one GPU (ranks as threads).

Each rank holds its row slab of B, Z and the mass lumps
(lgh_mat_create_rows with the in-process communicator of
lgh_rows_local_create); the library exchanges ghost rows once per product
and all-reduces every Gram, Q^T F Q, U^T X, residual norm and PCG dot
product.  No kernel waits for another rank: the ranks meet only on the
host, inside the communicator.  Against the one-rank build of the same
operators (the reference's MPI slabs give the same model, up to the
solves' tolerance, glr-woodbury-formulas.tex:76-98):

  - the sharded products equal the global CSR product rows;
  - sharded Z-solves (PCG, the block V-cycle plus the global coarse
    correction; or Jacobi) match
    the one-rank solves to the solve tolerance;
  - the sharded build keeps the same spectrum (1e-8 of lambda_max), the
    same logdet (1e-9) and the same solve / sample / apply (1e-7), in FP64
    and (against the FP64 sharded build) in mixed precision;
  - the incremental extend over slabs matches the one-rank extend;
  - every rank ends with the same spectrum;
  - the operations that do not run on slabs say so (LGH_ERR_SUP), and
    operators sharded differently are refused.
"""

import threading

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

pytestmark = pytest.mark.gpu

RTOL_Z = 1e-12


def _ranks(size, fn, timeout=600):
    """Run fn(rank, comm) on `size` threads with in-process row-slab
    communicators; returns the per-rank results (plain numpy values)."""
    comms = L.local_rows_comms(size)
    out, errs = [None] * size, []

    def body(r):
        try:
            out[r] = fn(r, comms[r])
        except Exception as e:                 # reported below
            errs.append((r, repr(e)))

    ts = [threading.Thread(target=body, args=(r,)) for r in range(size)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout)
    alive = any(t.is_alive() for t in ts)
    if not alive:
        L.free_local_rows_comms(comms)
    assert not alive, "a rank did not finish"
    assert not errs, errs
    return out


@pytest.fixture(scope="module")
def c1():
    return P.grid_problem("c1")


def petsc_split(N, size, r):
    """PETSc's default layout: N // size rows each, the remainder on the
    lowest ranks."""
    q, m = divmod(N, size)
    a = r * q + min(r, m)
    return a, a + q + (1 if r < m else 0)


def _slab(cfg, size, r, split=None):
    N = cfg["N"]
    a, b = (split or L.shard_range)(N, size, r)
    return a, b, L.rows_slab(cfg["B"], a, b), L.rows_slab(cfg["Z"], a, b)


@pytest.mark.parametrize("size", [2, 3])
def test_rows_products(cuda_device, c1, size):
    N = c1["N"]
    x = np.random.default_rng(1).standard_normal(N)
    yB = P.csr_matvec(c1["B"], x)
    yZ = P.csr_matvec(c1["Z"], x)

    def rank(r, comm):
        a, b, Bs, Zs = _slab(c1, size, r)
        Bm = L.Mat(Bs, rows=(N, comm))
        Zm = L.Mat(Zs, rows=(N, comm))
        row0, row1, ng = Bm.rows_info()
        assert (row0, row1) == (a, b) and ng > 0
        ex0 = Bm.rows_traffic()[0]
        yb = Bm.mult(x[a:b])
        zb = Zm.mult(x[a:b])
        assert Bm.rows_traffic()[0] == ex0 + 1
        return a, b, yb, zb

    for a, b, yb, zb in _ranks(size, rank):
        assert np.allclose(yb, yB[a:b], rtol=1e-13, atol=1e-13 * np.abs(yB).max())
        assert np.allclose(zb, yZ[a:b], rtol=1e-13, atol=1e-13 * np.abs(yZ).max())


@pytest.mark.parametrize("size,pc", [(2, None), (3, None), (2, "jacobi")])
def test_rows_zsolve_matches_one_rank(cuda_device, c1, size, pc):
    N, w = c1["N"], 12
    X = np.random.default_rng(2).standard_normal((N, w))
    opts = L.prior_opts(ksp_rtol=RTOL_Z)
    ref = L.Prior(Z=L.Mat(c1["Z"]), mass=c1["mass"], opts=opts, pc=pc)
    Y1 = ref.solve_block(X)

    def rank(r, comm):
        a, b, _, Zs = _slab(c1, size, r)
        pr = L.Prior(Z=L.Mat(Zs, rows=(N, comm)), mass=c1["mass"][a:b],
                     opts=opts, pc=pc)
        Y = pr.solve_block(X[a:b])
        y1 = pr.solve(X[a:b, 0])
        return a, b, Y, y1, pr.info()["mean_col_iters"]

    res = _ranks(size, rank)
    Y = np.concatenate([r[2] for r in res])
    y1 = np.concatenate([r[3] for r in res])
    err = np.linalg.norm(Y - Y1, axis=0) / np.linalg.norm(Y1, axis=0)
    assert err.max() < 1e-9, err.max()
    assert np.linalg.norm(y1 - Y1[:, 0]) < 1e-9 * np.linalg.norm(Y1[:, 0])
    # the residual of the assembled sharded solution, directly
    R = np.stack([P.csr_matvec(c1["Z"], Y[:, j]) for j in range(w)], 1) - X
    assert (np.linalg.norm(R, axis=0) / np.linalg.norm(X, axis=0)).max() < 1e-8
    its = [r[4] for r in res]
    assert len(set(its)) == 1          # every rank took the same iterations


def _glr_outputs(g, a, b, N, c=1.0):
    rng = np.random.default_rng(7)
    rhs, xi = rng.standard_normal(N), rng.standard_normal(N)
    return dict(lam=g.eigs().copy(), logdet=g.logdet(c),
                solve=g.solve(c, rhs[a:b]), sample=g.sample(c, xi[a:b]),
                apply=g.apply(c, rhs[a:b]), report=dict(g.report))


def _one_rank(cfg, gopts, exec=None, extend=0):
    N = cfg["N"]
    pr = L.Prior(Z=L.Mat(cfg["Z"]), mass=cfg["mass"],
                 opts=L.prior_opts(ksp_rtol=RTOL_Z))
    g = L.Glr(L.Mat(cfg["B"]), pr, gopts, exec=exec)
    if extend:
        g.extend(extend)
    return _glr_outputs(g, 0, N, N)


def _sharded(cfg, size, gopts, exec=None, extend=0, split=None):
    N = cfg["N"]

    def rank(r, comm):
        a, b, Bs, Zs = _slab(cfg, size, r, split)
        pr = L.Prior(Z=L.Mat(Zs, rows=(N, comm, a)), mass=cfg["mass"][a:b],
                     opts=L.prior_opts(ksp_rtol=RTOL_Z))
        Bm = L.Mat(Bs, rows=(N, comm, a))
        g = L.Glr(Bm, pr, gopts, exec=exec)
        if extend:
            g.extend(extend)
        out = _glr_outputs(g, a, b, N)
        out["traffic"] = Bm.rows_traffic()
        return out

    res = _ranks(size, rank)
    for r in res[1:]:                      # replicated on every rank
        assert np.array_equal(r["lam"], res[0]["lam"])
        assert r["logdet"] == res[0]["logdet"]
    out = dict(res[0])
    for k in ("solve", "sample", "apply"):
        out[k] = np.concatenate([r[k] for r in res])
    out["traffic"] = [r["traffic"] for r in res]
    return out


def _close(got, want, lam_tol=1e-8, vec_tol=1e-7):
    lw, lg = want["lam"], got["lam"]
    assert len(lg) == len(lw)
    assert np.abs(lg - lw).max() <= lam_tol * np.abs(lw).max()
    assert abs(got["logdet"] - want["logdet"]) <= 1e-9 * max(1., abs(want["logdet"]))
    for k in ("solve", "sample", "apply"):
        e = np.linalg.norm(got[k] - want[k]) / np.linalg.norm(want[k])
        assert e < vec_tol, (k, e)


@pytest.mark.parametrize("size", [2, 3])
def test_rows_build_matches_one_rank(cuda_device, c1, size):
    gopts = L.glr_opts(ell=c1["ell"], seed=11, trunc_rel=0.0)
    want = _one_rank(c1, gopts)
    got = _sharded(c1, size, gopts)
    _close(got, want)
    assert got["report"]["kept"] == want["report"]["kept"]
    # the Rayleigh-Ritz residual (about the first cut eigenvalue) is the
    # same quantity, computed from all-reduced partial norms
    rg, rw = got["report"]["resid_max"], want["report"]["resid_max"]
    assert abs(rg - rw) <= 1e-3 * rw + 1e-10 * np.abs(want["lam"]).max()
    for ex, nbytes, _ in got["traffic"]:
        assert ex > 0 and nbytes > 0


def test_rows_petsc_layout(cuda_device, c1):
    """Any contiguous split works, e.g. PETSc's MPIAIJ default (4096 rows on
    3 ranks: 1366, 1365, 1365, where the even split gives 1365, 1365,
    1366)."""
    assert petsc_split(c1["N"], 3, 0) != L.shard_range(c1["N"], 3, 0)
    gopts = L.glr_opts(ell=c1["ell"], seed=11, trunc_rel=0.0)
    want = _one_rank(c1, gopts)
    got = _sharded(c1, 3, gopts, split=petsc_split)
    _close(got, want)


def test_rows_bad_split_fails_on_every_rank(cuda_device, c1):
    """Rank 1 claims rows that leave a gap: every rank's creation fails
    (the ranks agree on the split before any exchange)."""
    N = c1["N"]

    def rank(r, comm):
        a, b = L.shard_range(N, 2, r)
        if r == 1:
            a += 8
        try:
            L.Mat(L.rows_slab(c1["B"], a, b), rows=(N, comm, a))
            return 0
        except L.LghError as e:
            return e.code

    assert _ranks(2, rank) == [62, 62]


def test_rows_extend_matches_one_rank(cuda_device, c1):
    gopts = L.glr_opts(ell=40, seed=5, trunc_rel=0.0)
    want = _one_rank(c1, gopts, extend=20)
    got = _sharded(c1, 2, gopts, extend=20)
    assert len(want["lam"]) > 40
    _close(got, want)


def test_rows_mixed_precision(cuda_device, c1):
    gopts = L.glr_opts(ell=c1["ell"], seed=11, trunc_rel=0.0)
    fp64 = _sharded(c1, 2, gopts)
    mixed = _sharded(c1, 2, gopts, exec=L.exec_opts(precision=L.PREC_MIXED))
    lam, lm = fp64["lam"], mixed["lam"]
    assert len(lm) == len(lam)
    assert np.abs(lm - lam).max() <= 1e-6 * np.abs(lam).max()
    e = np.linalg.norm(mixed["solve"] - fp64["solve"]) / np.linalg.norm(fp64["solve"])
    assert e < 1e-6


def test_rows_refusals(cuda_device, c1):
    N = c1["N"]

    def rank(r, comm):
        a, b, Bs, Zs = _slab(c1, 2, r)
        Bm = L.Mat(Bs, rows=(N, comm))
        Zm = L.Mat(Zs, rows=(N, comm))
        pr = L.Prior(Z=Zm, mass=c1["mass"][a:b],
                     opts=L.prior_opts(ksp_rtol=1e-10))
        # a replicated prior with a sharded B (and the reverse) is refused
        # on the host before any collective
        full = L.Prior(Z=L.Mat(c1["Z"]), mass=c1["mass"],
                       opts=L.prior_opts(ksp_rtol=1e-10))
        codes = []
        for Bx, px in ((Bm, full), (L.Mat(c1["B"]), pr)):
            try:
                L.Glr(Bx, px, L.glr_opts(ell=8, seed=1))
                codes.append(0)
            except L.LghError as e:
                codes.append(e.code)
        # Chebyshev modes need the global spectrum bounds: not on slabs
        try:
            L.Prior(Z=Zm, mass=c1["mass"][a:b],
                    opts=L.prior_opts(ksp_rtol=1e-10, blocked_mode=2))
            codes.append(0)
        except L.LghError as e:
            codes.append(e.code)
        g = L.Glr(Bm, pr, L.glr_opts(ell=16, seed=1, trunc_rel=0.0))
        R = np.ones((b - a, 2))
        try:
            g.solve_batch([1.0, 2.0], R)
            codes.append(0)
        except L.LghError as e:
            codes.append(e.code)
        try:
            L.Server(g)
            codes.append(0)
        except L.LghError as e:
            codes.append(e.code)
        return codes

    for codes in _ranks(2, rank):
        assert codes[0] == 62 and codes[1] == 62
        assert codes[2:] == [56] * 3, codes
