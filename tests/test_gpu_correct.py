"""The deflation correction (lgh_glr_correct_probes / lgh_glr_correct)
against the reference's own gates (tests/test_deflate.cpp), on the same
closed-form problem: N = 120, B SPD of exact rank 10 (the GLR model of B is
exact), diagonal Z and mass through prior callbacks, and a true Hessian
H_d = B + DH with a planted signed error of exact rank 4, so a correction
with enough probes / applies recovers F_true = whiten(H_d) exactly and every
claim is gated against a dense eigendecomposition of F_true.

  value pass: basis and apply accounting, no clamps, corrected signed
    spectrum == oracle, qc_before >> qc_after ~ 0, floor, logdet, the
    identity battery, extend and a second correction refused;
  fresh randomized: the same recovery through the sketch path;
  clamp: a large negative error mode makes H_d(c0) indefinite, the clamp
    engages and the corrected object stays consistent above its floor;
  threshold: d_keep_min above every priced |d| leaves the object
    uncorrected, still extendable and still correctable.
"""

import ctypes

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

pytestmark = pytest.mark.gpu

BACKENDS = [1, 0]          # LGH_GLR_REPLICATED, LGH_GLR_DEFAULT


def _rd(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _setup(err_scale, backend):
    p = P.test_deflate_problem(err_scale)
    z = p["zdiag"]

    def applyZ(x, y, ctx):
        vx = L.Vec(handle=ctypes.c_void_p(x))
        vy = L.Vec(handle=ctypes.c_void_p(y))
        vy.set(vx.get() * z)

    def solveZ(x, y, ctx):
        vx = L.Vec(handle=ctypes.c_void_p(x))
        vy = L.Vec(handle=ctypes.c_void_p(y))
        vy.set(vx.get() / z)

    B = L.Mat(dense=p["B_dense"])
    pr = L.Prior(mass=p["mass"], callbacks=dict(applyZ=applyZ, solveZ=solveZ))
    o = L.glr_opts(ell=40, q_power=1, trunc_abs=0., trunc_rel=1e-8,
                   backend=backend, nb=8, panel=16, check=0)
    g = L.Glr(B, pr, o)
    Hd = p["Hd"]
    return p, (B, pr), g, (lambda x: Hd @ x)


def _battery(g, c, v, tag):
    """corrected apply, solve, factor, sample and pow are mutually
    consistent actions of the same (U', lam') (test_deflate.cpp:215-250)"""
    y = g.apply(c, v)
    assert _rd(g.solve(c, y), v) < 1e-8, tag
    gt = g.factor(c, 1, v)
    assert _rd(g.factor(c, 0, gt), y) < 1e-8, tag
    ginvt = g.factor(c, 3, gt)
    assert _rd(ginvt, v) < 1e-8, tag
    assert _rd(g.sample(c, gt), ginvt) < 1e-14, tag
    assert _rd(g.pow(c, 1.0, g.pow(c, -1.0, v)), v) < 1e-10, tag


@pytest.mark.parametrize("backend", BACKENDS)
def test_value_pass(cuda_device, backend):
    c, k, n_qc = 0.7, 30, 6
    p, keep, g, hess = _setup(1.0, backend)
    V = p["probes"](k)
    HV = p["Hd"] @ V
    rep = g.correct_probes(V, HV, hess, L.correct_opts(c0=1.0, applies=8,
                                                       n_qc=n_qc))
    assert rep["basis"] == p["rank_c"]
    assert rep["hd_applies"] == p["rank_c"]
    assert rep["clamped"] == 0
    assert rep["qc_before"] > 1e-3
    assert rep["qc_after"] < 1e-7
    nk = p["rank_b"] + p["rank_c"]
    lam, orc = g.eigs(), p["oracle"][:nk]
    assert len(lam) == nk
    assert np.max(np.abs(lam - orc)) / abs(orc[0]) < 1e-7
    assert abs(rep["floor"] - max(0., -orc.min())) < 1e-8
    ref = float(np.sum(np.log(orc + c) - np.log(c)))
    assert abs(g.logdet(c) - ref) < 1e-8 * abs(ref)
    _battery(g, c, p["probe_vec"], "value pass")
    with pytest.raises(L.LghError) as e:
        g.extend(5)
    assert e.value.code == 58
    with pytest.raises(L.LghError) as e:
        g.correct_probes(V, HV, hess, L.correct_opts(c0=1.0, applies=8))
    assert e.value.code == 58


@pytest.mark.parametrize("backend", BACKENDS)
def test_fresh_randomized(cuda_device, backend):
    p, keep, g, hess = _setup(1.0, backend)
    rep = g.correct(hess, L.correct_opts(c0=1.0, applies=16))
    assert rep["basis"] == p["rank_c"]
    assert rep["clamped"] == 0
    nk = p["rank_b"] + p["rank_c"]
    lam, orc = g.eigs(), p["oracle"][:nk]
    assert len(lam) == nk
    assert np.max(np.abs(lam - orc)) / abs(orc[0]) < 1e-6
    _battery(g, 0.7, p["probe_vec"], "fresh")


@pytest.mark.parametrize("backend", BACKENDS)
def test_clamp(cuda_device, backend):
    c0, k = 1.0, 30
    p, keep, g, hess = _setup(400.0, backend)
    V = p["probes"](k)
    rep = g.correct_probes(V, p["Hd"] @ V, hess,
                           L.correct_opts(c0=c0, applies=8))
    eps = L.correct_opts().clamp_eps
    assert rep["clamped"] >= 1
    assert rep["floor"] < c0
    assert rep["d_min"] >= -1.0 + eps - 1e-12
    _battery(g, 2.0 * c0, p["probe_vec"], "clamp")


@pytest.mark.parametrize("backend", BACKENDS)
def test_threshold_leaves_object_uncorrected(cuda_device, backend):
    k = 30
    p, keep, g, hess = _setup(1.0, backend)
    V = p["probes"](k)
    HV = p["Hd"] @ V
    rep = g.correct_probes(V, HV, hess, L.correct_opts(c0=1.0, applies=8,
                                                       d_keep_min=10.0))
    assert rep["kept"] == 0
    assert rep["d_max"] != 0.
    assert len(g.eigs()) == p["rank_b"]
    g.extend(5)                              # still extendable
    rep = g.correct_probes(V, HV, hess, L.correct_opts(c0=1.0, applies=8))
    assert rep["kept"] > 0                   # and still correctable


def test_correct_argument_errors(cuda_device):
    p, keep, g, hess = _setup(1.0, 1)
    V = p["probes"](4)
    with pytest.raises(L.LghError) as e:
        g.correct_probes(V, p["Hd"] @ V, hess, L.correct_opts(n_qc=4))
    assert e.value.code == 63
    with pytest.raises(L.LghError) as e:
        g.correct(hess, L.correct_opts(applies=1))
    assert e.value.code == 63
    with pytest.raises(L.LghError) as e:
        g.correct(hess, L.correct_opts(c0=0.0))
    assert e.value.code == 63
