"""Saving and restoring a built GLR object (lgh_glr_save / lgh_glr_load):
the restored object serves the same spectrum, solves and samples without a
rebuild, extends incrementally from the saved sketch state to the same
spectrum as the original extended in memory, and a file for another size
or a corrupted file is refused."""

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_save_load_round_trip(cuda_device, tmp_path, precision):
    cfg = P.grid_problem("c1")
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-12))
    ex = L.exec_opts(precision=precision)
    g = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, trunc_rel=1e-3), exec=ex)
    path = tmp_path / "model.lgh"
    g.save(path, with_extension=True)
    h = L.Glr.load(B, pr, path)
    assert np.array_equal(g.eigs(), h.eigs())
    assert np.array_equal(g.U(), h.U())
    rhs = np.random.default_rng(2).standard_normal(cfg["N"])
    assert np.array_equal(g.solve(1.0, rhs), h.solve(1.0, rhs))
    assert np.array_equal(g.sample(0.5, rhs), h.sample(0.5, rhs))
    assert g.logdet(2.0) == h.logdet(2.0)
    # the loaded object continues the incremental extension
    g.extend(20)
    h.extend(20)
    lg, lh = g.eigs(), h.eigs()
    assert len(lg) == len(lh)
    assert np.max(np.abs(lg - lh)) <= 1e-12 * lg[0]


def test_load_rejects_wrong_size_and_corruption(cuda_device, tmp_path):
    cfg = P.grid_problem("c1")
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"])
    g = L.Glr(B, pr, L.glr_opts(ell=20, seed=0))
    path = tmp_path / "model.lgh"
    g.save(path)
    # no extension state saved: an incremental extend is refused
    h = L.Glr.load(B, pr, path)
    with pytest.raises(L.LghError) as e:
        h.extend(10)
    assert e.value.code == 73
    # another operator size
    tp = P.test_prior_mat_problem()
    Z2 = L.Mat(tp["Z"])
    pr2 = L.Prior(Z=Z2, mass=tp["mass"])
    B2 = L.Mat(P.diag_csr(np.ones(tp["n"])))
    with pytest.raises(L.LghError) as e:
        L.Glr.load(B2, pr2, path)
    assert e.value.code == 60
    # a flipped byte in U
    data = bytearray(path.read_bytes())
    data[len(data) // 2] ^= 0x40
    bad = tmp_path / "bad.lgh"
    bad.write_bytes(bytes(data))
    with pytest.raises(L.LghError) as e:
        L.Glr.load(B, pr, bad)
    assert e.value.code == 62
