"""The multigrid smoother's kernel (k_cheb, one Chebyshev-Jacobi step of a
CSR operator on a row-major block) against a numpy restatement of the step,
for every flag combination the V-cycle uses, in FP64 and FP32, on the 2D
5-point and 3D 7-point Z operators and on a matrix with rows of mixed
lengths, empty rows and rows without a diagonal entry (Jacobi scale 0).

One step: d_new = a d + b D^{-1} r (flags & 1: the a d term left out),
x += d_new (flags & 2: x taken as zero), r_new = r - A d_new, and d_new
stored (flags & 4).  And the two-step form the V-cycle runs at its default
degree (flags 8 and 16), bit for bit against two ordinary steps."""

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

pytestmark = pytest.mark.gpu

FLAGS = [L.CHEB_FIRST | L.CHEB_ZERO_X | L.CHEB_STORE_D,
         L.CHEB_FIRST | L.CHEB_STORE_D, L.CHEB_STORE_D, 0, L.CHEB_FIRST]


def _ragged(n=1500, seed=5):
    """Rows with 0..40 off-diagonal entries (longer than one 32-lane row
    group); every 7th row has no diagonal entry."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        k = int(rng.integers(0, 41))
        nb = rng.choice(np.delete(np.arange(n), i), size=k, replace=False)
        rows += [i] * k
        cols += list(nb)
        vals += list(0.1 * rng.standard_normal(k))
        if i % 7:
            rows.append(i)
            cols.append(i)
            vals.append(2.0 + rng.random())
    return P.coo_to_csr(n, np.array(rows), np.array(cols), np.array(vals))


@pytest.fixture(scope="module")
def ops(cuda_device):
    d = {
        "z2d": P.z_operator(48, 2, 25.0, P.lumped_mass(48, 2)),
        "z3d": P.z_operator(14, 3, 16.0, P.lumped_mass(14, 3)),
        "ragged": _ragged(),
    }
    return {k: (v, L.Mat(v)) for k, v in d.items()}


def _numpy_step(A, X, R, D, a, b, flags):
    Ad = P.csr_to_dense(A)
    diag = np.diag(Ad)
    dinv = np.where(diag != 0, 1.0 / np.where(diag != 0, diag, 1.0), 0.0)
    dn = b * dinv[:, None] * R
    if not flags & L.CHEB_FIRST:
        dn = dn + a * D
    x = dn if flags & L.CHEB_ZERO_X else X + dn
    return x, R - Ad @ dn, dn


@pytest.mark.parametrize("name", ["z2d", "z3d", "ragged"])
@pytest.mark.parametrize("fp32", [False, True])
def test_cheb_step_matches_numpy(ops, name, fp32):
    A, M = ops[name]
    n = A["n"]
    rng = np.random.default_rng(17)
    tol = 2e-5 if fp32 else 1e-12
    for w in (1, 3, 16, 60, 220):
        X = rng.standard_normal((n, w))
        R = rng.standard_normal((n, w))
        D = rng.standard_normal((n, w))
        if fp32:
            X, R, D = (v.astype(np.float32).astype(np.float64) for v in (X, R, D))
        for fl in FLAGS:
            a, b = 0.37, 0.81
            x1, r1, d1 = L.test_cheb_step(M, X, R, D, a, b, fl, fp32)
            xe, re, de = _numpy_step(A, X, R, D, a, b, fl)
            assert np.abs(x1 - xe).max() <= tol * (1 + np.abs(xe).max()), (w, fl)
            assert np.abs(r1 - re).max() <= tol * (1 + np.abs(re).max()), (w, fl)
            if fl & L.CHEB_STORE_D:
                assert np.abs(d1 - de).max() <= tol * (1 + np.abs(de).max())
            # deterministic: the same call gives the same bits
            x2, r2, _ = L.test_cheb_step(M, X, R, D, a, b, fl, fp32)
            assert np.array_equal(x1, x2) and np.array_equal(r1, r2)


def test_cheb_step_column_slices_same_bits(ops, monkeypatch):
    """An operator whose neighbour band would not fit the L2 budget is swept
    in column slices; the slices give the same bits as one sweep."""
    A, M = ops["z3d"]
    n = A["n"]
    rng = np.random.default_rng(23)
    X, R, D = (rng.standard_normal((n, 220)) for _ in range(3))
    out = {}
    for budget in ("0", "0.05"):     # never slice / slice into many
        monkeypatch.setenv("LGH_CHEB_L2MB", budget)
        out[budget] = [L.test_cheb_step(M, X, R, D, 0.37, 0.81, fl)
                       for fl in FLAGS]
    for a, b in zip(out["0"], out["0.05"]):
        for u, v in zip(a, b):
            assert np.array_equal(u, v)


@pytest.mark.parametrize("name", ["z2d", "z3d", "ragged"])
@pytest.mark.parametrize("fp32", [False, True])
def test_two_step_pair_same_bits(ops, name, fp32):
    """The smoother's two-step form (the V-cycle's default degree): a first
    step that stores only its residual (flags 8), then a step that forms
    the first step's d and x from that step's input residual (flags 16,
    coefficient bp), gives the same bits as two ordinary steps, from x = 0
    (pre-smoothing) and from a given x (post-smoothing)."""
    A, M = ops[name]
    n = A["n"]
    rng = np.random.default_rng(23)
    b1, a2, b2 = 0.93, 0.41, 1.27
    for w in (1, 3, 16, 60, 220):
        X = rng.standard_normal((n, w))
        R0 = rng.standard_normal((n, w))
        if fp32:
            X, R0 = (v.astype(np.float32).astype(np.float64) for v in (X, R0))
        zero = np.zeros_like(R0)
        for zx in (L.CHEB_ZERO_X, 0):
            # two ordinary steps
            x1, r1, d1 = L.test_cheb_step(M, X, R0, zero, 0.0, b1,
                                          L.CHEB_FIRST | zx | L.CHEB_STORE_D,
                                          fp32)
            x2, r2, _ = L.test_cheb_step(M, x1, r1, d1, a2, b2, 0, fp32)
            # the pair: residual only, then the step that forms d1 and x1
            xs, s1, _ = L.test_cheb_step(M, X, R0, zero, 0.0, b1,
                                         L.CHEB_FIRST | zx | L.CHEB_R_ONLY,
                                         fp32)
            assert np.array_equal(xs, X)            # x left untouched
            assert np.array_equal(s1, r1), (w, zx)
            y2, s2, _ = L.test_cheb_step(M, X, s1, R0, a2, b2,
                                         L.CHEB_PREV_R | zx, fp32, bp=b1)
            assert np.array_equal(y2, x2), (w, zx)
            assert np.array_equal(s2, r2), (w, zx)
