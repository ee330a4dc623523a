"""Mixed precision (LGH_PREC_MIXED: FP32 sketch blocks, F-applies and
CholQR2 sweeps with FP64 accumulation; Z-solves with FP64 Krylov vectors
and an FP32 V-cycle; FP64 small dense work, eigenvectors and downstream
operations) against the plain FP64 build on the same inputs and the same
hashed sketch.  The reference computes in FP64 only;
the mixed form is an extension whose accuracy is reported against FP64:
eigenvalue error relative to the largest eigenvalue, the largest principal
angle between the leading eigenvector subspaces, and solve / logdet
agreement.
"""

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

pytestmark = pytest.mark.gpu

MIXED = 1


@pytest.fixture(scope="module")
def c1(cuda_device):
    cfg = P.grid_problem("c1")
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-12))
    return cfg, B, Z, pr


def _sin_max(U1, U2):
    s = np.linalg.svd(U2.T @ U1, compute_uv=False)
    return float(np.sqrt(max(0.0, 1.0 - np.min(s) ** 2)))


def test_mixed_spectrum_matches_fp64(c1):
    cfg, B, Z, pr = c1
    o = L.glr_opts(ell=60, seed=0, trunc_rel=1e-3)
    g64 = L.Glr(B, pr, o)
    g32 = L.Glr(B, pr, o, exec=L.exec_opts(precision=MIXED))
    assert g32.stats()["precision"] == MIXED
    l64, l32 = g64.eigs(), g32.eigs()
    k = min(len(l64), len(l32)) - 1
    assert k >= 20
    assert abs(len(l64) - len(l32)) <= 1
    err = np.max(np.abs(l32[:k] - l64[:k])) / l64[0]
    assert err < 1e-6, err
    # leading, well separated eigenvectors span the same subspace
    U64, U32 = g64.U()[:, :10], g32.U()[:, :10]
    assert _sin_max(U64, U32) < 1e-3
    # downstream operations run in FP64 on the mixed model
    rhs = np.random.default_rng(4).standard_normal(cfg["N"])
    x64, x32 = g64.solve(1.0, rhs), g32.solve(1.0, rhs)
    assert np.linalg.norm(x32 - x64) / np.linalg.norm(x64) < 1e-4
    ld64, ld32 = g64.logdet(1.0), g32.logdet(1.0)
    assert abs(ld32 - ld64) < 1e-4 * abs(ld64)


def test_mixed_extend_equals_one_shot(c1):
    """Incremental extension in mixed precision (FP32 BCGS2 against the old
    basis) reaches the one-shot mixed spectrum at the extended width."""
    cfg, B, Z, pr = c1
    ex = L.exec_opts(precision=MIXED)
    ga = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, trunc_rel=1e-3), exec=ex)
    ga.extend(20)
    gb = L.Glr(B, pr, L.glr_opts(ell=60, seed=0, trunc_rel=1e-3), exec=ex)
    la, lb = ga.eigs(), gb.eigs()
    k = min(len(la), len(lb)) - 1
    assert k >= 20
    assert np.max(np.abs(la[:k] - lb[:k])) / lb[0] < 1e-6


def test_mixed_batch_solves_reach_fp64_accuracy(c1):
    """The batched solves of a mixed object run FP64 PCG with the FP32
    V-cycle as preconditioner to the prior's tolerance (1e-12 here), so
    they agree with the FP64 single-vector solve of the same model to FP64
    solver accuracy."""
    cfg, B, Z, pr = c1
    g = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, check=0),
              exec=L.exec_opts(precision=MIXED))
    before = pr.info()
    R = np.random.default_rng(9).standard_normal((cfg["N"], 2))
    cs = [0.1, 3.0]
    X = g.solve_batch(cs, R)
    after = pr.info()
    assert after["pc32_calls"] >= before["pc32_calls"] + 3  # W, y1, y0
    for si, c in enumerate(cs):
        for j in range(2):
            ref = g.solve(c, R[:, j])
            assert np.linalg.norm(X[si][:, j] - ref) \
                < 1e-8 * np.linalg.norm(ref)
    S = g.sample_batch(cs, R)
    for si, c in enumerate(cs):
        ref = g.sample(c, R[:, 0])
        assert np.linalg.norm(S[si][:, 0] - ref) < 1e-8 * np.linalg.norm(ref)


def test_mixed_many_shift_batch_on_tensor_cores(c1):
    """A mixed-precision object's many-shift batch runs its combination on
    tcgen05 (TF32 in three passes, FP32 accumulation): 9 shifts x 64
    right-hand sides (576 output columns: several 128- and 256-column
    tiles), 4096 rows (32 row tiles), up to 60 kept modes (two 32-value K
    stages).  Against the FP64 single-vector operations of the same model:
    relative error below 1e-6 (about FP32 accuracy on the correction term,
    which is small beside f(c) y0 here)."""
    cfg, B, Z, pr = c1
    g = L.Glr(B, pr, L.glr_opts(ell=60, seed=0, trunc_rel=1e-6, check=0),
              exec=L.exec_opts(precision=MIXED))
    assert len(g.eigs()) > 32
    R = np.random.default_rng(21).standard_normal((cfg["N"], 64))
    cs = np.logspace(-3, 3, 9)
    for rep in range(2):                      # tuning call, then the graph
        X = g.solve_batch(cs, R)
        S = g.sample_batch(cs, R)
        info = g.batch_info()
        assert info["variant"] in (2, 3, 4, 5), info
        for si in (0, 4, 8):
            for j in (0, 63):
                ref = g.solve(cs[si], R[:, j])
                assert np.linalg.norm(X[si][:, j] - ref) \
                    < 1e-6 * np.linalg.norm(ref), (rep, si, j)
                refs = g.sample(cs[si], R[:, j])
                assert np.linalg.norm(S[si][:, j] - refs) \
                    < 1e-6 * np.linalg.norm(refs), (rep, si, j)
    assert info["replays"] >= 1
