"""The multigrid set-up's host products, on the CPU.

The smoothed-aggregation hierarchy is built on the host with OpenMP
(csrc/mg.cu): aggregation, the smoothed prolongator P, R = P^T by an
order-preserving parallel transpose, A P and P^T (A P) by two-pass
Gustavson products, and the symmetrisation of the Galerkin operator
against each entry's mirror.  Through lgh_test_mg_galerkin, which runs the
first coarsening with no device call, these tests check that:
  * the result is the same bits for 1 and 4 threads (every host reduction
    and product sums in a fixed order);
  * Ac equals the symmetrised P^T A P of scipy to 1e-14 relative, and is
    exactly symmetric;
  * P has the coarse size's columns and no empty row;
  * a malformed CSR is refused with an error, not read out of bounds.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import lgh_b200 as L
from lgh_b200 import problems as P


def _sp(c):
    return sp.csr_matrix((c["vals"], c["colidx"], c["rowptr"]),
                         shape=(c["n"], c["m"]))


def _same_bits(a, b):
    return (np.array_equal(a["rowptr"], b["rowptr"])
            and np.array_equal(a["colidx"], b["colidx"])
            and np.array_equal(a["vals"].view(np.int64),
                               b["vals"].view(np.int64)))


@pytest.mark.parametrize("name", ["c1", "c2", "c3_32"])
def test_galerkin_independent_of_threads_and_exact(name):
    Z = P.grid_problem(name)["Z"]
    n = len(Z["rowptr"]) - 1
    zc = dict(n=n, rowptr=Z["rowptr"], colidx=Z["colidx"], vals=Z["vals"])
    P1, A1 = L.test_mg_galerkin(zc, threads=1)
    P4, A4 = L.test_mg_galerkin(zc, threads=4)
    assert _same_bits(P1, P4) and _same_bits(A1, A4)

    nc = A1["n"]
    assert 1 < nc < n and P1["m"] == nc
    assert np.all(np.diff(P1["rowptr"]) > 0)          # no empty row of P
    Zs = sp.csr_matrix((Z["vals"], Z["colidx"], Z["rowptr"]), shape=(n, n))
    Ps, Acs = _sp(P1), _sp(A1)
    ref = Ps.T @ (Zs @ Ps)
    ref = 0.5 * (ref + ref.T)
    err = sp.linalg.norm(Acs - ref) / sp.linalg.norm(ref)
    assert err < 1e-14, err
    asym = (Acs - Acs.T).tocsr()
    asym.eliminate_zeros()
    assert asym.nnz == 0                               # exactly symmetric


def test_galerkin_refuses_malformed_csr():
    rp = np.array([0, 2, 1, 3], dtype=np.int64)       # not monotone
    ci = np.array([0, 1, 2], dtype=np.int32)
    with pytest.raises(L.LghError):
        L.test_mg_galerkin(dict(n=3, rowptr=rp, colidx=ci,
                                vals=np.ones(3)))
    rp = np.array([0, 1, 2, 3], dtype=np.int64)
    ci = np.array([0, 1, 7], dtype=np.int32)          # column out of range
    with pytest.raises(L.LghError):
        L.test_mg_galerkin(dict(n=3, rowptr=rp, colidx=ci,
                                vals=np.ones(3)))
