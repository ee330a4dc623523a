"""The request loop (lgh_server_*): continuous batching of solve / sample /
logdet requests over a resident GLR object, checked against the library's
own single-request operations (lgh_glr_solve_batch / _sample_batch /
lgh_glr_logdet, themselves checked against the oracle in test_gpu_glr.py).

The loop runs every request column through its own CG state inside a shared
slot block, so a request's result must not depend on what it was batched
with: the same request alone and inside a mix gives the same bits.
"""

import numpy as np
import pytest

import lgh_b200 as L
import lgh_b200.problems as P

pytestmark = pytest.mark.gpu


def _rd(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def c1(cuda_device):
    cfg = P.grid_problem("c1")
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-12))
    g = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, check=0))
    return cfg, (B, Z, pr), g


def _reqs(n, seed):
    rng = np.random.default_rng(seed)
    return [
        (L.Server.SOLVE, 1.0, rng.standard_normal((n, 3))),
        (L.Server.SAMPLE, 0.5, rng.standard_normal((n, 2))),
        (L.Server.LOGDET, 2.0, None),
        (L.Server.SOLVE, 10.0, rng.standard_normal((n, 1))),
        (L.Server.SAMPLE, 1e-2, rng.standard_normal((n, 5))),
        (L.Server.SOLVE, 1e-3, rng.standard_normal((n, 4))),
    ]


def test_server_matches_batched_ops(c1):
    cfg, keep, g = c1
    n = cfg["N"]
    sv = L.Server(g, slots=16)
    reqs = _reqs(n, 5)
    ids = [sv.submit(k, c, X) for k, c, X in reqs]
    outs = [sv.wait(i) for i in ids]
    for (k, c, X), (y, lat) in zip(reqs, outs):
        assert lat > 0.
        if k == L.Server.LOGDET:
            assert abs(y - g.logdet(c)) == 0.0
            continue
        ref = (g.solve_batch if k == L.Server.SOLVE else g.sample_batch)(
            [c], X)[0]
        for j in range(X.shape[1]):
            assert _rd(y[:, j], ref[:, j]) < 1e-8, (k, c, j)
    st = sv.stats()
    assert st["completed"] == len(reqs)
    assert st["columns"] == sum(X.shape[1] for _, _, X in reqs
                                if X is not None)
    assert 0. < st["p50_s"] <= st["p99_s"] <= st["max_s"]
    assert st["pending"] == 0
    sv.close()


def test_server_result_independent_of_batch(c1):
    cfg, keep, g = c1
    n = cfg["N"]
    rng = np.random.default_rng(11)
    Xa = rng.standard_normal((n, 2))
    Xs = rng.standard_normal((n, 3))
    sv = L.Server(g, slots=16)
    alone = sv.wait(sv.submit(L.Server.SOLVE, 0.3, Xa))[0]
    alone_s = sv.wait(sv.submit(L.Server.SAMPLE, 0.3, Xs))[0]
    # the same requests in a mix, submitted behind and between others
    others = _reqs(n, 6)
    ids = [sv.submit(k, c, X) for k, c, X in others[:3]]
    ia = sv.submit(L.Server.SOLVE, 0.3, Xa)
    ids += [sv.submit(k, c, X) for k, c, X in others[3:]]
    isam = sv.submit(L.Server.SAMPLE, 0.3, Xs)
    mixed = sv.wait(ia)[0]
    mixed_s = sv.wait(isam)[0]
    for i in ids:
        sv.wait(i)
    assert np.array_equal(alone, mixed)
    assert np.array_equal(alone_s, mixed_s)
    sv.close()


def test_server_more_columns_than_slots_queue(c1):
    """Requests whose columns exceed the free slots wait in arrival order
    and run as slots free up."""
    cfg, keep, g = c1
    n = cfg["N"]
    rng = np.random.default_rng(3)
    sv = L.Server(g, slots=4)
    blocks = [rng.standard_normal((n, m)) for m in (4, 3, 4, 1, 2)]
    ids = [sv.submit(L.Server.SOLVE, 1.0, X) for X in blocks]
    for i, X in zip(ids, blocks):
        y = sv.wait(i)[0]
        ref = g.solve_batch([1.0], X)[0]
        assert _rd(y, ref) < 1e-8
    assert sv.stats()["completed"] == len(blocks)
    sv.close()


def test_server_argument_errors(c1):
    cfg, keep, g = c1
    n = cfg["N"]
    sv = L.Server(g, slots=4)
    with pytest.raises(L.LghError) as e:
        sv.submit(L.Server.SOLVE, 1.0, np.ones((n, 0)))   # m = 0
    assert e.value.code == 60
    with pytest.raises(L.LghError) as e:
        sv.submit(L.Server.SOLVE, -1.0, np.ones((n, 1)))  # c <= floor
    assert e.value.code == 63
    with pytest.raises(L.LghError) as e:
        sv.submit(7, 1.0, np.ones((n, 1)))
    assert e.value.code == 63
    sv.close()


def test_server_request_wider_than_slots(c1):
    """A request with more columns than the slot block runs in parts and
    gives the same bits as its columns submitted one at a time."""
    cfg, keep, g = c1
    n = cfg["N"]
    rng = np.random.default_rng(21)
    X = rng.standard_normal((n, 11))
    Xs = rng.standard_normal((n, 9))
    sv = L.Server(g, slots=4)
    wide = sv.wait(sv.submit(L.Server.SOLVE, 0.7, X))[0]
    wide_s = sv.wait(sv.submit(L.Server.SAMPLE, 0.7, Xs))[0]
    ref = g.solve_batch([0.7], X)[0]
    ref_s = g.sample_batch([0.7], Xs)[0]
    assert _rd(wide, ref) < 1e-8
    assert _rd(wide_s, ref_s) < 1e-8
    one = np.column_stack([sv.wait(sv.submit(L.Server.SOLVE, 0.7,
                                             X[:, j:j + 1]))[0]
                           for j in range(X.shape[1])])
    assert np.array_equal(one, wide)
    sv.close()


@pytest.fixture(scope="module")
def c1_mixed(cuda_device):
    cfg = P.grid_problem("c1")
    B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
    pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=1e-12))
    g = L.Glr(B, pr, L.glr_opts(ell=40, seed=0, check=0),
              exec=L.exec_opts(precision=L.PREC_MIXED))
    return cfg, (B, Z, pr), g


def test_server_mixed_object(c1_mixed):
    """A mixed-precision object's loop runs FP32 V-cycles under FP64 CG:
    its results agree with the object's own batched operations to the
    Z-solve tolerance and stay independent of the batch."""
    cfg, keep, g = c1_mixed
    n = cfg["N"]
    reqs = _reqs(n, 9)
    sv = L.Server(g, slots=8)
    ids = [sv.submit(k, c, X) for k, c, X in reqs]
    outs = [sv.wait(i)[0] for i in ids]
    for (k, c, X), y in zip(reqs, outs):
        if k == L.Server.LOGDET:
            assert abs(y - g.logdet(c)) == 0.0
            continue
        ref = (g.solve_batch if k == L.Server.SOLVE else g.sample_batch)(
            [c], X)[0]
        assert _rd(y, ref) < 1e-8, (k, c)
    k, c, X = reqs[0]
    alone = sv.wait(sv.submit(k, c, X))[0]
    assert np.array_equal(alone, outs[0])
    sv.close()
