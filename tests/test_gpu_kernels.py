"""Kernel-level parity on the GPU, through the C ABI's test hooks.

Each device kernel against the oracle (the CPU restatement of the
reference) or an FP64 LAPACK/numpy computation of the same quantity:
  sketch     integer xorshift state bit-exact; values within 2 ulp (the
             device log and glibc's log may round differently)
  spmm       CSR x row-major block, FP64 rel < 1e-14, FP32 rel < 1e-5
  zsolve     blocked PCG / Chebyshev vs a dense solve, the reference's
             tolerances (tests/test_prior_mat.cpp:141-190)
  gram/gemm  rel < 1e-13
  potrf      vs numpy Cholesky, jitter retry and double failure
  syev       Jacobi vs LAPACK eigenvalues, rel to ||A|| < 1e-13
"""

import json
import os

import numpy as np
import pytest

import lgh_b200 as L
import oracle
from lgh_b200 import problems as P

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(autouse=True)
def _dev(cuda_device):
    L.load()


def _rd(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_rng_state_bit_exact():
    for seed, j0 in [(271828, 0), (0, 200), (0xB0BD5, 0), (2 ** 63 + 5, 17)]:
        st = L.test_rng_state(seed, 300, j0, 9)
        for i in range(0, 300, 37):
            for j in range(9):
                assert int(st[i, j]) == oracle.lib().orc_rng_state_at(
                    seed, i, j0 + j)


def test_sketch_matches_reference_kat():
    with open(os.path.join(HERE, "golden", "rng_kat.json")) as f:
        d = json.load(f)
    ref = np.array([[float.fromhex(x) for x in row] for row in d["block"]])
    dev = L.test_sketch(d["block_seed"], 64, 0, 8)
    ulp = np.abs(dev - ref) / np.spacing(np.abs(ref))
    assert np.max(ulp) <= 2.0
    for e in d["kat"]:
        if e["i"] > 5000:
            continue
        v = L.test_sketch(int(e["seed"]), e["i"] + 1, e["j"], 1)[e["i"], 0]
        r = float.fromhex(e["value"])
        assert abs(v - r) <= 2 * np.spacing(abs(r)), e


def test_sketch_matches_oracle_block():
    n, j0, k = 5000, 37, 13
    dev = L.test_sketch(271828, n, j0, k)
    ref = oracle.sketch(271828, n, j0, k)
    ulp = np.abs(dev - ref) / np.spacing(np.abs(ref))
    assert np.max(ulp) <= 2.0
    assert np.mean(dev == ref) > 0.9


@pytest.mark.parametrize("w", [1, 3, 8, 16, 61, 220])
def test_spmm_fp64(w):
    cfg = P.grid_problem("c1")
    A = L.Mat(cfg["B"])
    X = np.random.default_rng(w).standard_normal((cfg["N"], w))
    Y = L.test_spmm(A, X)
    ref = P.csr_matvec(cfg["B"], X)
    assert _rd(Y, ref) < 1e-14


@pytest.mark.parametrize("w", [1, 16, 200])
def test_spmm_fp32(w):
    cfg = P.grid_problem("c1")
    A = L.Mat(cfg["B"])
    X = np.random.default_rng(w).standard_normal((cfg["N"], w))
    Y = L.test_spmm(A, X, fp32=True)
    ref = P.csr_matvec(cfg["B"], X)
    assert _rd(Y, ref) < 1e-5


@pytest.mark.parametrize("R", [0, 2, 4, 8])
@pytest.mark.parametrize("w", [8, 33, 64, 220])
def test_strip_product_fp64(R, w):
    """The strip form of B (k_strip.cu) against the CSR product, on the 2D
    config-1 kernel matrix and on a 3D one (config 3's formulas on 32^3)."""
    for name in ("c1", "c3_32"):
        cfg = P.grid_problem(name)
        A = L.Mat(cfg["B"])
        X = np.random.default_rng(w + R).standard_normal((cfg["N"], w))
        Y, used = L.test_spmm_strip(A, X, R=R)
        assert used in (2, 4, 8) and (R == 0 or used == R)
        ref = P.csr_matvec(cfg["B"], X)
        assert _rd(Y, ref) < 1e-14, (name, R, w)


@pytest.mark.parametrize("w", [8, 200])
def test_strip_product_fp32(w):
    cfg = P.grid_problem("c1")
    A = L.Mat(cfg["B"])
    X = np.random.default_rng(w).standard_normal((cfg["N"], w))
    Y, _ = L.test_spmm_strip(A, X, fp32=True)
    ref = P.csr_matvec(cfg["B"], X)
    assert _rd(Y, ref) < 1e-5


def test_strip_product_unsorted_rows_and_duplicates():
    """Rows whose columns are shuffled, duplicated entries and a ragged
    last strip: every stored entry is used exactly once."""
    rng = np.random.default_rng(5)
    n = 1003                                   # not a multiple of 8
    rows, cols, vals = [], [], []
    for i in range(n):
        nb = int(rng.integers(0, 12))
        cs = np.clip(i + rng.integers(-30, 31, size=nb), 0, n - 1)
        if i % 7 == 0 and nb:                  # a duplicated entry
            cs = np.concatenate([cs, cs[:1]])
        rng.shuffle(cs)
        rows += [i] * len(cs)
        cols += list(cs)
        vals += list(rng.standard_normal(len(cs)))
    rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
    order = np.argsort(rows, kind="stable")    # CSR order, columns unsorted
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr)
    csr = dict(n=n, rowptr=rowptr, colidx=cols[order].astype(np.int32),
               vals=vals[order])
    A = L.Mat(csr)
    X = rng.standard_normal((n, 40))
    ref = np.zeros((n, 40))
    np.add.at(ref, rows, vals[:, None] * X[cols])
    for R in (2, 4, 8):
        Y, _ = L.test_spmm_strip(A, X, R=R)
        assert np.max(np.abs(Y - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def _prior_mat(mode, tile=8, rtol=1e-12, pc="jacobi"):
    p = P.test_prior_mat_problem()
    Z = L.Mat(p["Z"])
    pr = L.Prior(Z=Z, mass=p["mass"],
                 opts=L.prior_opts(blocked_mode=mode, tile=tile,
                                   ksp_rtol=rtol), pc=pc)
    return p, Z, pr


@pytest.mark.parametrize("mode,pc", [(0, "jacobi"), (2, "jacobi"),
                                     (0, "amg"), (2, "amg"), (3, "amg")])
def test_zsolve_prior_mat_gates(mode, pc):
    """tests/test_prior_mat.cpp:141-190 on the device, for the Jacobi and
    the multigrid preconditioner (blocked modes 0, 2, 3)"""
    p, Z, pr = _prior_mat(mode, pc=pc)
    Zd = P.csr_to_dense(p["Z"])
    b = p["probe"]
    xref = np.linalg.solve(Zd, b)
    assert _rd(pr.solve(b), xref) < 1e-8
    X = np.stack([b * (1 + 0.1 * j) for j in range(11)], 1)
    Y = pr.solve_block(X)
    worst = max(_rd(Y[:, j] / (1 + 0.1 * j), xref) for j in range(11))
    assert worst < 1e-7
    zb = Z.mult(b)
    assert _rd(pr.solve(zb), b) < 1e-8


def test_cheb_bounds_match_oracle():
    p, Z, pr = _prior_mat(2)
    info = pr.info()
    Zo = oracle.Csr(p["Z"]["rowptr"], p["Z"]["colidx"], p["Z"]["vals"])
    po = oracle.Prior(Zo, p["mass"], mode=2, tile=8)
    oi = po.info()
    assert abs(info["emin"] - oi["emin"]) < 1e-8 * oi["emax"]
    assert abs(info["emax"] - oi["emax"]) < 1e-8 * oi["emax"]
    assert abs(info["nit"] - oi["nit"]) <= 1


@pytest.mark.parametrize("w", [1, 5, 64])
def test_zsolve_pcg_c1_vs_oracle(w):
    cfg = P.grid_problem("c1")
    Z = L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-10),
                 pc="jacobi")
    X = np.random.default_rng(3).standard_normal((cfg["N"], w))
    Y = L.test_zsolve(pr, X)
    Zo = oracle.Csr(cfg["Z"]["rowptr"], cfg["Z"]["colidx"], cfg["Z"]["vals"])
    po = oracle.Prior(Zo, cfg["mass"], ksp_rtol=1e-10)
    Yo = po.solve_block(X)
    Zd = P.csr_to_dense(cfg["Z"])
    ref = np.linalg.solve(Zd, X)
    for j in range(w):
        assert _rd(Y[:, j], ref[:, j]) < 1e-8
        assert _rd(Y[:, j], Yo[:, j]) < 1e-8
    # per-column iteration counts match the oracle's CG
    assert abs(pr.info()["mean_col_iters"] - po.info()["mean_cg_its"]) <= 2


@pytest.mark.parametrize("nu", [1, 2, 3])
def test_zsolve_amg_smoother_degrees(nu):
    """The V-cycle at smoother degrees 1 to 3, FP64 and FP32.  Degree 2 (the
    default) runs the two-step form: a residual-only first step, the post
    residual r2 - (A P) x_c and the prolongation fused into the
    post-smoothing pass; the other degrees run the plain step sequence with
    direction blocks.  Each solves to the dense answer, and a higher degree
    takes no more PCG iterations than a lower one."""
    cfg = P.grid_problem("c1")
    Z = L.Mat(cfg["Z"])
    X = np.random.default_rng(11).standard_normal((cfg["N"], 16))
    ref = np.linalg.solve(P.csr_to_dense(cfg["Z"]), X)
    its = {}
    for k in sorted({1, nu}):
        pr = L.Prior(Z=Z, mass=cfg["mass"],
                     opts=L.prior_opts(ksp_rtol=1e-10, nu_force=k))
        assert pr.info()["mg_levels"] >= 2
        Y = L.test_zsolve(pr, X)
        assert max(_rd(Y[:, j], ref[:, j]) for j in range(16)) < 1e-8
        its[k] = pr.info()["mean_col_iters"]
        pr32 = L.Prior(Z=Z, mass=cfg["mass"],
                       opts=L.prior_opts(ksp_rtol=1e-5, nu_force=k))
        Y32 = L.test_zsolve(pr32, X, fp32=True)
        assert max(_rd(Y32[:, j], ref[:, j]) for j in range(16)) < 1e-3
    assert its[nu] <= its[1]


def test_zsolve_fp32():
    cfg = P.grid_problem("c1")
    Z = L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-5))
    X = np.random.default_rng(4).standard_normal((cfg["N"], 16))
    Y = L.test_zsolve(pr, X, fp32=True)
    ref = np.linalg.solve(P.csr_to_dense(cfg["Z"]), X)
    assert max(_rd(Y[:, j], ref[:, j]) for j in range(16)) < 1e-3


def test_zsolve_columns_independent():
    """A column's result does not depend on the other columns of its block
    (each column has its own CG scalars and convergence mask): the same
    column solved alone or inside a 12-wide block agrees to rounding (the
    lane grouping, and so the reduction tree, changes with the width), and
    a rerun of the same shape is bitwise identical."""
    cfg = P.grid_problem("c1")
    Z = L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-10))
    X = np.random.default_rng(5).standard_normal((cfg["N"], 12))
    Yall = L.test_zsolve(pr, X)
    Y1 = L.test_zsolve(pr, X[:, 3:4])
    assert _rd(Y1[:, 0], Yall[:, 3]) < 1e-12
    X2 = X.copy()
    X2[:, 5] *= 1e3                      # a much larger neighbour column
    Y3 = L.test_zsolve(pr, X2)
    assert _rd(Y3[:, 3], Yall[:, 3]) < 1e-12
    Y2 = L.test_zsolve(pr, X)
    assert np.array_equal(Yall, Y2)


@pytest.mark.parametrize("n,w", [(1000, 1), (5000, 40), (70000, 220)])
def test_gram(n, w):
    X = np.random.default_rng(n).standard_normal((n, w))
    G = L.test_gram(X)
    ref = X.T @ X
    assert np.max(np.abs(G - ref)) < 1e-13 * np.max(np.abs(ref)) * 10
    assert np.array_equal(G, G.T)


def test_gemm_nn():
    rng = np.random.default_rng(9)
    X = rng.standard_normal((30001, 77))
    M = rng.standard_normal((77, 45))
    Y = L.test_gemm_nn(X, M)
    assert _rd(Y, X @ M) < 1e-14


@pytest.mark.parametrize("n", [1, 7, 40, 220, 413])
def test_potrf_trtri(n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n + 5, n))
    G = A.T @ A
    Lc, Li, info = L.test_potrf(G)
    assert info[0] == 0 and info[1] == 0
    ref = np.linalg.cholesky(G)
    assert np.max(np.abs(Lc - ref)) < 1e-11 * np.max(np.abs(ref))
    assert np.max(np.abs(Li @ Lc - np.eye(n))) < 1e-9


def test_potrf_jitter_and_failure():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((40, 10))
    G = A @ A.T                                       # rank 10 of 40
    Lc, Li, info = L.test_potrf(G, jitter_mode=0)
    if info[1]:
        # the replicated rule: + 1e-12 tr(G)/n on the diagonal
        Gj = G + 1e-12 * np.trace(G) / 40 * np.eye(40)
        assert info[0] == 0
        assert np.max(np.abs(Lc @ Lc.T - Gj)) < 1e-10 * np.max(np.abs(G))
    Lc, Li, info = L.test_potrf(-np.eye(5))
    assert info[0] == 1 and info[1] == 1


@pytest.mark.parametrize("n", [2, 3, 40, 41, 220])
def test_syev_jacobi(n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    A = (A + A.T) / 2
    w, V, sweeps = L.test_syev(A)
    ref = np.linalg.eigvalsh(A)
    assert np.max(np.abs(np.sort(w) - ref)) < 1e-13 * np.linalg.norm(A)
    assert np.max(np.abs(V.T @ V - np.eye(n))) < 1e-12
    assert np.max(np.abs(A @ V - V * w)) < 1e-12 * np.linalg.norm(A)
    assert 1 <= sweeps <= 40


def test_syev_graded_spectrum():
    """Eigenvalues spanning 12 decades keep relative accuracy."""
    rng = np.random.default_rng(0)
    n = 60
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.logspace(0, -12, n) * np.where(np.arange(n) % 3 == 0, -1, 1)
    A = (Q * lam) @ Q.T
    A = (A + A.T) / 2
    w, V, _ = L.test_syev(A)
    ref = np.linalg.eigvalsh(A)
    top = np.argsort(-np.abs(ref))[:20]
    rs = np.sort(ref[top])
    ws = np.sort(w[np.argsort(-np.abs(w))[:20]])
    assert np.max(np.abs(ws - rs) / np.abs(rs)) < 1e-10


@pytest.mark.parametrize("w", [1, 7, 64])
@pytest.mark.parametrize("mode", [0, 3])
def test_zsolve_amg_c1(w, mode):
    """The multigrid-preconditioned Z-solve (CG + V-cycle, the reference's
    CG + PCGAMG; and Chebyshev around the V-cycle, its mode 3) against a
    dense solve on config 1; it converges in few iterations."""
    cfg = P.grid_problem("c1")
    Z = L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"],
                 opts=L.prior_opts(ksp_rtol=1e-10, blocked_mode=mode,
                                   tile=0), pc="amg")
    info0 = pr.info()
    assert info0["mg_levels"] >= 2 and info0["mg_coarse"] <= 1500
    X = np.random.default_rng(8).standard_normal((cfg["N"], w))
    Y = L.test_zsolve(pr, X)
    ref = np.linalg.solve(P.csr_to_dense(cfg["Z"]), X)
    worst = max(_rd(Y[:, j], ref[:, j]) for j in range(w))
    assert worst < 1e-8
    info = pr.info()
    if mode == 0:
        assert info["mean_col_iters"] < 60
    else:
        assert info["nit"] < 60


def test_zsolve_amg_c2_shape():
    """config-2 operator (N = 262144): the hierarchy coarsens to a dense
    level and the V-cycle CG meets rtol 1e-10 in a few tens of iterations,
    checked by the FP64 residual."""
    cfg = P.grid_problem("c2")
    Z = L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-10),
                 pc="amg")
    X = np.random.default_rng(9).standard_normal((cfg["N"], 4))
    Y = L.test_zsolve(pr, X)
    R = X - P.csr_matvec(cfg["Z"], Y)
    for j in range(4):
        assert np.linalg.norm(R[:, j]) / np.linalg.norm(X[:, j]) < 1e-7
    assert pr.info()["mean_col_iters"] < 80
