"""GLR build and downstream operations on the GPU, through the C ABI.

* The reference's gates (tests/test_glr.cpp, N = 120, exact rank 10) with
  its tolerances, for the Mat-path prior and the callbacks prior, SPD and
  indefinite B, incremental and replicated extension.
* Parity with the oracle on the same inputs (same seed, same sketch):
  spectra, solve / sample outputs, logdet.
* test_prior_mat.cpp's end-to-end gate with a Chebyshev (mode 2) prior.
* Batched operations against the single-vector ones, error codes.
"""

import ctypes
import json
import os

import numpy as np
import pytest

import lgh_b200 as L
import oracle
from lgh_b200 import problems as P

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
C = 0.7


@pytest.fixture(autouse=True)
def _dev(cuda_device):
    L.load()


def _rd(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _dense_ref(spd):
    with open(os.path.join(HERE, "golden", "dense_spectra.json")) as f:
        d = json.load(f)["spectra"]
    return np.array([float.fromhex(x) for x in
                     d["test_glr_spd" if spd else "test_glr_indef"]])


def _opts(ell=40, **kw):
    return L.glr_opts(ell=ell, q_power=1, trunc_abs=0., trunc_rel=1e-8, nb=8,
                      panel=16, check=1, **kw)


def _callback_prior(p):
    """diagonal Z through user callbacks (tests/test_glr.cpp:61-85)"""
    z = p["zdiag"]

    def applyZ(x, y, ctx):
        vx, vy = L.Vec(handle=ctypes.c_void_p(x)), L.Vec(
            handle=ctypes.c_void_p(y))
        vy.set(vx.get() * z)

    def solveZ(x, y, ctx):
        vx, vy = L.Vec(handle=ctypes.c_void_p(x)), L.Vec(
            handle=ctypes.c_void_p(y))
        vy.set(vx.get() / z)

    return L.Prior(mass=p["mass"], callbacks=dict(applyZ=applyZ,
                                                  solveZ=solveZ))


def _setup(spd, path):
    p = P.test_glr_problem(spd=spd)
    B = L.Mat(dense=p["B_dense"])
    if path == "mat":
        Z = L.Mat(p["Z"])
        pr = L.Prior(Z=Z, mass=p["mass"])
        keep = (B, Z, pr)
    else:
        pr = _callback_prior(p)
        keep = (B, pr)
    return p, B, pr, keep


@pytest.mark.parametrize("path", ["mat", "callbacks"])
@pytest.mark.parametrize("spd", [True, False])
def test_glr_reference_gates(spd, path):
    p, B, pr, keep = _setup(spd, path)
    g = L.Glr(B, pr, _opts())
    rep = g.report
    dense = _dense_ref(spd)
    lam = g.eigs()
    assert rep["kept"] == 10
    assert np.max(np.abs(lam - np.abs(dense[:10])) / np.abs(dense[:10])) < 1e-8
    assert rep["next_abs"] < 1e-6 * rep["lam_abs_max"]
    assert rep["resid_max"] < 1e-7 * rep["lam_abs_max"]
    if not spd:
        assert rep["n_negative_raw"] >= 5
    ref = np.sum(np.log(np.abs(dense[:10]) + C) - np.log(C))
    assert abs(g.logdet(C) - ref) < 1e-9 * abs(ref)
    if spd:
        v = p["probe"]
        y = g.apply(C, v)
        assert _rd(g.solve(C, y), v) < 1e-8
        x = g.factor(C, 1, v)
        assert _rd(g.factor(C, 0, x), y) < 1e-8
        yy = g.factor(C, 1, v)
        x = g.factor(C, 3, yy)
        assert _rd(x, v) < 1e-8
        assert _rd(g.sample(C, yy), x) < 1e-14
        assert _rd(g.pow(C, 1.0, g.pow(C, -1.0, v)), v) < 1e-10
        fl = 1.0 / np.sqrt(lam + C)
        assert _rd(g.filter(fl, 1 / np.sqrt(C), v), g.pow(C, -0.5, v)) < 1e-12
        x = g.factor(C, 2, y)                       # GINV(G(.)) identity
        assert _rd(g.factor(C, 0, x), y) < 1e-8


@pytest.mark.parametrize("backend", [0, 1])
@pytest.mark.parametrize("spd", [True, False])
def test_extend_equals_one_shot(spd, backend):
    """extend(10) from ell=30 == one-shot ell=40 (tests/test_glr.cpp:299-316);
    backend 0 = incremental (BCGS2 + bordered T), 1 = replicated rebuild"""
    p, B, pr, keep = _setup(spd, "mat")
    g = L.Glr(B, pr, _opts(backend=backend))
    g2 = L.Glr(B, pr, _opts(ell=30, backend=backend))
    g2.extend(10)
    l1, l2 = g.eigs(), g2.eigs()
    assert len(l1) == len(l2)
    assert np.max(np.abs(l1 - l2) / np.abs(l1)) < 1e-10


def test_extend_to_400_on_40k_rows():
    """Incremental extension 200 -> 400 on a 200^2 grid (40000 rows: enough
    rows that the split-K products run at their full split count, so every
    BCGS2 panel product needs its largest partial-sum workspace), against
    the one-shot build at ell = 400."""
    n, dim = 200, 2
    mass = P.lumped_mass(n, dim)
    Z = L.Mat(P.z_operator(n, dim, 25.0, mass))
    B = L.Mat(P.b_operator(n, dim, 0.01, 0.03, mass,
                           P.a_field(n, dim, "sincos")))
    pr = L.Prior(Z=Z, mass=mass, opts=L.prior_opts(ksp_rtol=1e-12))
    g1 = L.Glr(B, pr, L.glr_opts(ell=400, seed=0, trunc_rel=0.0, check=0))
    g2 = L.Glr(B, pr, L.glr_opts(ell=200, seed=0, trunc_rel=0.0, check=0))
    g2.extend(200)
    l1, l2 = g1.eigs()[:100], g2.eigs()[:100]
    assert np.max(np.abs(l1 - l2) / np.abs(l1)) < 1e-9


@pytest.mark.parametrize("spd", [True, False])
def test_parity_with_oracle_test_glr(spd):
    p, B, pr, keep = _setup(spd, "mat")
    g = L.Glr(B, pr, _opts())
    Bo = oracle.Csr(p["B"]["rowptr"], p["B"]["colidx"], p["B"]["vals"])
    Zo = oracle.Csr(p["Z"]["rowptr"], p["Z"]["colidx"], p["Z"]["vals"])
    po = oracle.Prior(Zo, p["mass"])
    go = oracle.Glr(Bo, po, oracle.opts_default(
        ell=40, q_power=1, trunc_abs=0., trunc_rel=1e-8, nb=8, panel=16,
        check=1))
    assert g.report["kept"] == go.report["kept"]
    assert np.max(np.abs(g.eigs() - go.eigs()) / go.eigs()) < 1e-12
    for k in ("lam_abs_max", "lam_raw_min", "lam_raw_max"):
        assert abs(g.report[k] - go.report[k]) < 1e-12 * go.report["lam_abs_max"]
    # n_negative_raw also counts the ell - rank noise-level eigenvalues,
    # whose signs are rounding; the reference gates only the indefinite
    # case's count (tests/test_glr.cpp:241-243)
    if not spd:
        assert g.report["n_negative_raw"] >= 5 and go.report["n_negative_raw"] >= 5
    assert abs(g.logdet(C) - go.logdet(C)) < 1e-13 * abs(go.logdet(C))
    v = p["probe"]
    if spd:
        assert _rd(g.solve(C, v), go.solve(C, v)) < 1e-12
        assert _rd(g.sample(C, v), go.sample(C, v)) < 1e-12


def test_prior_mat_end_to_end_mode2():
    """tests/test_prior_mat.cpp:221-277 with a Chebyshev (mode 2) prior"""
    p = P.test_prior_mat_problem()
    Z = L.Mat(p["Z"])
    pr = L.Prior(Z=Z, mass=p["mass"], opts=L.prior_opts(blocked_mode=2,
                                                        tile=8), pc="jacobi")
    B = L.Mat(dense=p["B_dense"])
    g = L.Glr(B, pr, L.glr_opts(ell=16, trunc_rel=1e-6, backend=1))
    assert g.report["kept"] == 6
    v = p["probe"]
    assert _rd(g.solve(C, g.apply(C, v)), v) < 1e-6


def _c1(ell=60, rank_cap=None):
    cfg = P.grid_problem("c1")
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-12))
    return cfg, (B, Z, pr)


def test_c1_parity_with_oracle():
    """Config 1 (64^2 grid, ell = 60, q = 1, seed 0) against the oracle on
    the same inputs: same sketch, same algorithm; Z-solves to rtol 1e-12
    on both sides, so spectra agree to solver accuracy."""
    cfg, (B, Z, pr) = _c1()
    o = L.glr_opts(ell=60, seed=0, trunc_rel=1e-3)
    g = L.Glr(B, pr, o)
    Bo = oracle.Csr(cfg["B"]["rowptr"], cfg["B"]["colidx"], cfg["B"]["vals"])
    Zo = oracle.Csr(cfg["Z"]["rowptr"], cfg["Z"]["colidx"], cfg["Z"]["vals"])
    po = oracle.Prior(Zo, cfg["mass"], ksp_rtol=1e-12)
    go = oracle.Glr(Bo, po, oracle.opts_default(ell=60, seed=0,
                                                trunc_rel=1e-3))
    ld, lo = g.eigs(), go.eigs()
    assert len(ld) == len(lo)
    assert np.max(np.abs(ld - lo) / lo) < 1e-8
    assert abs(g.logdet(1.0) - go.logdet(1.0)) < 1e-9 * abs(go.logdet(1.0))
    rhs = oracle.sketch(1, cfg["N"], 0, 1)[:, 0]
    assert _rd(g.solve(1.0, rhs), go.solve(1.0, rhs)) < 1e-7
    assert _rd(g.sample(1.0, rhs), go.sample(1.0, rhs)) < 1e-7
    # the eigen-residual of a truncated (not exact-rank) sketch is a property
    # of the problem: the device and the oracle report the same figure
    assert abs(g.report["resid_max"] - go.report["resid_max"]) \
        < 1e-3 * go.report["resid_max"]


def test_batch_matches_single():
    cfg, keep = _c1()
    B, Z, pr = keep
    g = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, check=0))
    rng = np.random.default_rng(2)
    R = rng.standard_normal((cfg["N"], 3))
    cs = np.array([1e-2, 1.0, 30.0])
    Xs = g.solve_batch(cs, R)
    Ss = g.sample_batch(cs, R)
    for si, c in enumerate(cs):
        for j in range(3):
            assert _rd(Xs[si][:, j], g.solve(c, R[:, j])) < 1e-8
            assert _rd(Ss[si][:, j], g.sample(c, R[:, j])) < 1e-8
    ld = g.logdet_batch(cs)
    for si, c in enumerate(cs):
        assert abs(ld[si] - g.logdet(c)) <= 1e-14 * abs(ld[si])


def test_many_shift_batch_graph_replay():
    """Many shifts in one fused combination, captured as a graph on the
    first call of a shape and replayed on the next: the replay writes the
    new call's output buffer with the new call's shifts.  Both calls match
    the single-vector operations."""
    cfg, keep = _c1()
    B, Z, pr = keep
    g = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, check=0))
    rng = np.random.default_rng(12)
    R = rng.standard_normal((cfg["N"], 5))
    cs1 = np.logspace(-3, 3, 7)
    cs2 = np.logspace(-2, 2, 7) * 1.5
    X1 = g.solve_batch(cs1, R)
    info1 = g.batch_info()
    X2 = g.solve_batch(cs2, R)
    info2 = g.batch_info()
    assert info1["tuned_shapes"] >= 1 and info1["variant"] in (0, 1)
    assert info2["captures"] == max(info1["captures"], 1)
    assert info2["replays"] == info1["replays"] + 1
    for cs, X in ((cs1, X1), (cs2, X2)):
        for si in (0, 3, 6):
            for j in (0, 4):
                assert _rd(X[si][:, j], g.solve(cs[si], R[:, j])) < 1e-8
    S = g.sample_batch(cs2, R)
    for si in (0, 6):
        assert _rd(S[si][:, 1], g.sample(cs2[si], R[:, 1])) < 1e-8


def test_single_shift_batch_before_and_after_w():
    """One shift on an object without W = Z^{-1} M^{1/2} U takes the
    per-call formula (no W); once W exists (a multi-shift call builds it)
    the same call goes through W.  Both agree with the single-vector
    operations."""
    cfg, keep = _c1()
    B, Z, pr = keep
    g = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, check=0))
    rng = np.random.default_rng(4)
    R = rng.standard_normal((cfg["N"], 5))
    c = 0.3
    x_direct = g.solve_batch([c], R)[0]
    s_direct = g.sample_batch([c], R)[0]
    g.solve_batch([c, 2 * c], R[:, :1])          # builds W
    x_w = g.solve_batch([c], R)[0]
    s_w = g.sample_batch([c], R)[0]
    for j in range(R.shape[1]):
        ref = g.solve(c, R[:, j])
        refs = g.sample(c, R[:, j])
        assert _rd(x_direct[:, j], ref) < 1e-8
        assert _rd(x_w[:, j], ref) < 1e-8
        assert _rd(s_direct[:, j], refs) < 1e-8
        assert _rd(s_w[:, j], refs) < 1e-8


def test_sample_covariance_is_inverse_model_hessian():
    """x = G^{-T} xi has covariance H~(c)^{-1} exactly: the linear map S of
    sample satisfies S S^T = H~(c)^{-1} with H~ = Z M^{-1/2}(U L U^T + cI)
    M^{-1/2} Z (docs/glr-woodbury-formulas.tex:45-56)."""
    p = P.test_glr_problem(spd=True)
    B = L.Mat(dense=p["B_dense"])
    Z = L.Mat(p["Z"])
    pr = L.Prior(Z=Z, mass=p["mass"])
    g = L.Glr(B, pr, _opts())
    n = p["n"]
    S = np.stack([g.sample(C, e) for e in np.eye(n)], 1)
    U = g.U()
    lam = g.eigs()
    zs = p["zdiag"] / np.sqrt(p["mass"])
    Ht = zs[:, None] * ((U * lam) @ U.T + C * np.eye(n)) * zs[None, :]
    assert np.max(np.abs(S @ S.T @ Ht - np.eye(n))) < 1e-8
    # and a sampling check: 4000 draws, covariance of projections
    rng = np.random.default_rng(11)
    Xi = rng.standard_normal((n, 4000))
    X = S @ Xi
    probes = rng.standard_normal((n, 4))
    emp = np.cov(probes.T @ X)
    exact = probes.T @ np.linalg.inv(Ht) @ probes
    assert np.max(np.abs(emp - exact) / np.sqrt(np.outer(np.diag(exact),
                                                          np.diag(exact)))) \
        < 0.12


def test_deterministic_rebuild():
    cfg, (B, Z, pr) = _c1()
    o = L.glr_opts(ell=30, seed=5, check=0)
    l1 = L.Glr(B, pr, o).eigs()
    l2 = L.Glr(B, pr, o).eigs()
    assert np.array_equal(l1, l2)


def test_error_codes():
    p, B, pr, keep = _setup(True, "mat")
    with pytest.raises(L.LghError) as e:
        L.Glr(B, pr, _opts(ell=121))
    assert e.value.code == 63
    g = L.Glr(B, pr, _opts())
    with pytest.raises(L.LghError) as e:
        g.solve(0.0, p["probe"])
    assert e.value.code == 63
    with pytest.raises(L.LghError) as e:
        g.extend(0)
    assert e.value.code == 63
    with pytest.raises(L.LghError) as e:
        g.extend(200)
    assert e.value.code == 63
    v = L.Vec(data=p["probe"])
    rc = L.load().lgh_glr_solve(g.h, C, v.h, v.h)
    assert rc == 62
    Lb = L.load()
    h = ctypes.c_void_p()
    assert Lb.lgh_prior_create_ksp(None, v.h, None, ctypes.byref(h)) == 56


def test_treatments():
    p = P.test_glr_problem(spd=False)
    B = L.Mat(dense=p["B_dense"])
    Z = L.Mat(p["Z"])
    pr = L.Prior(Z=Z, mass=p["mass"])
    dense = _dense_ref(False)
    flip = L.Glr(B, pr, _opts(treat=0)).eigs()
    relu = L.Glr(B, pr, _opts(treat=1)).eigs()
    none = L.Glr(B, pr, _opts(treat=2)).eigs()
    assert np.allclose(flip, np.abs(dense[:10]), rtol=1e-8)
    assert np.allclose(none, dense[:10], rtol=1e-8)
    assert np.allclose(relu, np.maximum(dense[:10], 0), rtol=1e-8, atol=0)
