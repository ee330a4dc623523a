"""The oracle pinned to the reference's own code (CPU).

rng_kat.json holds known answers of the reference's lgh_randn_at and
lgh_zs_cheb_count compiled from the reference source (oracle/build_ref.sh;
tests/golden/gen_golden.py).  The oracle restatement must reproduce them
bit for bit; where the reference build is present in this tree the two
are also compared directly on a sweep of (seed, i, j).
"""

import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def _kat():
    with open(os.path.join(HERE, "golden", "rng_kat.json")) as f:
        return json.load(f)


def test_randn_at_matches_reference_kat():
    d = _kat()
    for e in d["kat"]:
        v = oracle.randn_at(int(e["seed"]), e["i"], e["j"])
        assert float(v).hex() == e["value"], e
        st = oracle.lib().orc_rng_state_at(int(e["seed"]), e["i"], e["j"])
        assert format(st, "016x") == e["state"], e


def test_sketch_block_matches_reference_kat():
    d = _kat()
    blk = oracle.sketch(d["block_seed"], 64, 0, 8)
    ref = np.array([[float.fromhex(x) for x in row] for row in d["block"]])
    assert np.array_equal(blk, ref)


def test_cheb_count_matches_reference_kat():
    for e in _kat()["cheb_count"]:
        assert oracle.lib().orc_cheb_count(e["lmin"], e["lmax"], e["tol"]) \
            == e["nit"]


def test_randn_at_direct_against_reference_build():
    ref = oracle.ref_pure()
    if ref is None:
        pytest.skip("reference build (oracle/_ref) not present on this host")
    rng = np.random.default_rng(7)
    for _ in range(3000):
        s = int(rng.integers(0, 2 ** 63))
        i = int(rng.integers(0, 3_000_000))
        j = int(rng.integers(0, 2048))
        assert oracle.randn_at(s, i, j) == ref.ref_randn_at(s, i, j)


def test_dense_spectra_fixture_consistent():
    from lgh_b200 import problems as P
    with open(os.path.join(HERE, "golden", "dense_spectra.json")) as f:
        d = json.load(f)["spectra"]
    for spd in (True, False):
        p = P.test_glr_problem(spd=spd)
        s = np.sqrt(p["mass"]) / p["zdiag"]
        F = s[:, None] * p["B_dense"] * s[None, :]
        w, _ = oracle.dsyevd(F)
        w = w[np.argsort(-np.abs(w), kind="stable")][:10]
        ref = np.array([float.fromhex(x) for x in
                        d["test_glr_spd" if spd else "test_glr_indef"]])[:10]
        assert np.max(np.abs(w - ref) / np.abs(ref)) < 1e-12
