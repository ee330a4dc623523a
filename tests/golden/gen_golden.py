"""Generate the committed golden fixtures (run where the reference tree is).

* rng_kat.json: known answers of the reference's OWN lgh_randn_at and
  lgh_zs_cheb_count (include/lgpsf_hessian/impl/glr_common_impl.h:32-73,
  zsolve_impl.h:93-102), compiled from the reference source by
  oracle/build_ref.sh into oracle/_ref/liblgh_ref_pure.so.  Values are
  stored as float.hex strings (bit-exact).
* dense_spectra.json: the dense-LAPACK oracle spectra of the reference's
  gate problems (tests/test_glr.cpp:91-123: F = M^{1/2} Z^{-1} B Z^{-T}
  M^{1/2} formed densely, dsyevd, |lambda|-descending), computed with
  numpy's LAPACK from the closed-form entries.

Usage: python tests/golden/gen_golden.py   (from the repository root)
"""

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(
    __file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "lgpsf-hessian_b200"))

import oracle  # noqa: E402
from lgh_b200 import problems as P  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (seed, i, j) triples: edge rows/columns, large indices, the sketch seeds
# of the reference's defaults (271828), its Z-probe seed (0xB0BD5), seed 0,
# and a seed with the top bit set.
SEEDS = [0, 1, 271828, 0xB0BD5, 2 ** 63 + 12345, 2 ** 64 - 1]
IJ = [(0, 0), (1, 0), (0, 1), (119, 39), (4095, 59), (262143, 219),
      (884735, 399), (2097151, 519), (12345, 200), (12345, 201),
      (7, 1000), (2 ** 31 - 2, 3)]


def main():
    ref = oracle.ref_pure()
    if ref is None:
        raise SystemExit("oracle/_ref/liblgh_ref_pure.so missing: run "
                         "make -C oracle (needs the reference tree)")
    kat = []
    for s in SEEDS:
        for i, j in IJ:
            v = ref.ref_randn_at(s, i, j)
            st = oracle.lib().orc_rng_state_at(s, i, j)
            kat.append(dict(seed=str(s), i=i, j=j, value=float(v).hex(),
                            state=format(st, "016x")))
    # a dense block: 64 rows x 8 columns at seed 271828
    block = [[float(ref.ref_randn_at(271828, i, j)).hex() for j in range(8)]
             for i in range(64)]
    cheb = []
    for lmin, lmax, tol in [(0.1157172521511829, 2.070067612618547, 1e-10),
                            (0.9, 4.4, 1e-10), (1e-3, 2.0, 1e-8),
                            (0.5, 8.5, 1e-12)]:
        cheb.append(dict(lmin=lmin, lmax=lmax, tol=tol,
                         nit=int(ref.ref_cheb_count(lmin, lmax, tol))))
    with open(os.path.join(HERE, "rng_kat.json"), "w") as f:
        json.dump(dict(source="reference lgh_randn_at / lgh_zs_cheb_count "
                              "compiled by oracle/build_ref.sh",
                       kat=kat, block_seed=271828, block=block,
                       cheb_count=cheb), f, indent=1)

    spectra = {}
    for spd in (True, False):
        p = P.test_glr_problem(spd=spd)
        s = np.sqrt(p["mass"]) / p["zdiag"]
        F = s[:, None] * p["B_dense"] * s[None, :]
        w = np.linalg.eigvalsh(F)
        w = w[np.argsort(-np.abs(w), kind="stable")]
        spectra["test_glr_spd" if spd else "test_glr_indef"] = \
            [float(x).hex() for x in w[:20]]
    with open(os.path.join(HERE, "dense_spectra.json"), "w") as f:
        json.dump(dict(source="dense F of tests/test_glr.cpp:91-123, "
                              "numpy LAPACK eigvalsh, |lambda|-descending",
                       spectra=spectra), f, indent=1)
    print("wrote", os.path.join(HERE, "rng_kat.json"), "and dense_spectra.json")


if __name__ == "__main__":
    main()
