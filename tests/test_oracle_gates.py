"""The reference's own gates, run on the oracle (CPU).

tests/test_glr.cpp (N = 120, exact rank 10, diagonal Z, dense-LAPACK
oracle) and tests/test_prior_mat.cpp (24 x 24 Laplacian + 0.5 I), with the
reference's tolerances.  These pin the oracle before it is trusted as the
checker of the CUDA path.
"""

import json
import os

import numpy as np
import pytest

import oracle
from lgh_b200 import problems as P

HERE = os.path.dirname(os.path.abspath(__file__))
C = 0.7


def _dense_ref(spd):
    with open(os.path.join(HERE, "golden", "dense_spectra.json")) as f:
        d = json.load(f)["spectra"]
    return np.array([float.fromhex(x) for x in
                     d["test_glr_spd" if spd else "test_glr_indef"]])


def _rd(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _build(spd, ell=40, incremental=True):
    p = P.test_glr_problem(spd=spd)
    B = oracle.Csr(p["B"]["rowptr"], p["B"]["colidx"], p["B"]["vals"])
    Z = oracle.Csr(p["Z"]["rowptr"], p["Z"]["colidx"], p["Z"]["vals"])
    pr = oracle.Prior(Z, p["mass"])
    o = oracle.opts_default(ell=ell, q_power=1, trunc_abs=0., trunc_rel=1e-8,
                            nb=8, panel=16, check=1)
    return p, (B, Z, pr), oracle.Glr(B, pr, o, incremental=incremental)


@pytest.mark.parametrize("spd", [True, False])
def test_glr_gates_oracle(spd):
    p, keep, g = _build(spd)
    rep = g.report
    dense = _dense_ref(spd)
    lam = g.eigs()
    assert rep["kept"] == 10                                   # :221
    assert np.max(np.abs(lam - np.abs(dense[:10])) / np.abs(dense[:10])) \
        < 1e-8                                                 # :222-232
    assert rep["next_abs"] < 1e-6 * rep["lam_abs_max"]         # :233-234
    assert rep["resid_max"] < 1e-7 * rep["lam_abs_max"]        # :235-237
    if not spd:
        assert rep["n_negative_raw"] >= 5                      # :241-243
    ref = np.sum(np.log(np.abs(dense[:10]) + C) - np.log(C))
    assert abs(g.logdet(C) - ref) < 1e-9 * abs(ref)            # :245-252
    if spd:
        v = p["probe"]
        y = g.apply(C, v)
        assert _rd(g.solve(C, y), v) < 1e-8                    # :258-261
        x = g.factor(C, 1, v)
        assert _rd(g.factor(C, 0, x), y) < 1e-8                # :264-267
        yy = g.factor(C, 1, v)
        x = g.factor(C, 3, yy)
        assert _rd(x, v) < 1e-8                                # :270-274
        assert _rd(g.sample(C, yy), x) < 1e-14                 # :275-277
        assert _rd(g.pow(C, 1.0, g.pow(C, -1.0, v)), v) < 1e-10  # :280-283
        fl = 1.0 / np.sqrt(lam + C)
        assert _rd(g.filter(fl, 1 / np.sqrt(C), v), g.pow(C, -0.5, v)) \
            < 1e-12                                            # :286-296


@pytest.mark.parametrize("spd", [True, False])
@pytest.mark.parametrize("incremental", [False, True])
def test_extend_equals_one_shot_oracle(spd, incremental):
    _, keep, g = _build(spd)
    _, keep2, g2 = _build(spd, ell=30, incremental=incremental)
    g2.extend(10)
    l1, l2 = g.eigs(), g2.eigs()
    assert len(l1) == len(l2)                                  # :311
    assert np.max(np.abs(l1 - l2) / np.abs(l1)) < 1e-10        # :312-314


@pytest.mark.parametrize("mode", [0, 2])
def test_prior_mat_gates_oracle(mode):
    p = P.test_prior_mat_problem()
    Zd = P.csr_to_dense(p["Z"])
    b = p["probe"]
    xref = np.linalg.solve(Zd, b)
    Z = oracle.Csr(p["Z"]["rowptr"], p["Z"]["colidx"], p["Z"]["vals"])
    pr = oracle.Prior(Z, p["mass"], mode=mode, tile=8)
    x, _ = pr.solveZ(b)
    assert _rd(x, xref) < 1e-8                                 # :141-144
    X = np.stack([b * (1 + 0.1 * j) for j in range(11)], 1)
    Y = pr.solve_block(X)
    worst = max(_rd(Y[:, j] / (1 + 0.1 * j), xref) for j in range(11))
    assert worst < 1e-7                                        # :146-182
    x, _ = pr.solveZ(pr.applyZ(b))
    assert _rd(x, b) < 1e-8                                    # :185-190
    if mode == 2:
        B = oracle.Csr(p["B"]["rowptr"], p["B"]["colidx"], p["B"]["vals"])
        g = oracle.Glr(B, pr, oracle.opts_default(ell=16, trunc_rel=1e-6))
        assert g.report["kept"] == 6                           # :262
        v = p["probe"]
        assert _rd(g.solve(C, g.apply(C, v)), v) < 1e-6        # :267-270


def test_oracle_c1_shape_runs():
    """Config 1 sizes (64^2 grid) build on the oracle with the stated rank."""
    cfg = P.grid_problem("c1")
    assert cfg["N"] == 4096
    nnz_row = cfg["nnz_B"] / cfg["N"]
    assert 100 < nnz_row < 120                       # stated ~113 nnz/row
    B = oracle.Csr(cfg["B"]["rowptr"], cfg["B"]["colidx"], cfg["B"]["vals"])
    Z = oracle.Csr(cfg["Z"]["rowptr"], cfg["Z"]["colidx"], cfg["Z"]["vals"])
    pr = oracle.Prior(Z, cfg["mass"], ksp_rtol=1e-10)
    g = oracle.Glr(B, pr, oracle.opts_default(ell=24, seed=0, check=0,
                                              trunc_rel=1e-3))
    lam = g.eigs()
    assert len(lam) > 0 and np.all(np.diff(lam) <= 0)


def test_build_in_pieces_equals_one_shot():
    """The oracle's build advanced in bounded pieces (7-column F-apply
    waves) is the same object, bit for bit, as the one-shot build; the
    piece count matches the plan; the rank cap keeps the largest |lambda|
    and reports the first cut mode as next_abs."""
    p, (B, Z, pr), g = _build(True)
    o = oracle.opts_default(ell=40, q_power=1, trunc_abs=0., trunc_rel=1e-8,
                            nb=8, panel=16, check=1)
    b = oracle.Build(B, pr, o, wave=7)
    steps = 1
    while b.step():
        steps += 1
    gp = b.finish()
    assert steps == oracle.build_pieces(40, 1, gp.report["kept"], 7)
    assert np.array_equal(gp.eigs(), g.eigs())
    assert np.array_equal(gp.U(), g.U())
    assert gp.report["resid_max"] == g.report["resid_max"]
    v = p["probe"]
    assert np.array_equal(gp.solve(C, v), g.solve(C, v))
    X = np.stack([v, 2 * v + 1], axis=1)
    Xs = gp.solve_block(C, X)
    for j in range(2):
        x1 = g.solve(C, X[:, j])
        assert _rd(Xs[:, j], x1) < 1e-13
    gc = oracle.Glr(B, pr, o, cap=6)
    assert gc.report["kept"] == 6
    assert np.array_equal(gc.eigs(), g.eigs()[:6])
    assert gc.report["next_abs"] == g.eigs()[6]
