"""Run one device case of the GLR path through the C ABI (profiling driver).

  python lgpsf-hessian_b200/lgh_b200/kcase.py zsolve c2 220 [rtol] [fp32]
  python lgpsf-hessian_b200/lgh_b200/kcase.py spmm   c2 220
  python lgpsf-hessian_b200/lgh_b200/kcase.py build  c2 220

zsolve: blocked Z-solve of a seeded N x w block (PCG, Jacobi) with the
prior of the named configuration; spmm: B times a seeded N x w block;
build: one GLR build at ell = w.  Prints the wall time and the library's
per-kernel event timing.  Used for ncu captures of single kernels on the
benchmark's shapes.
"""

import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

import lgh_b200 as L  # noqa: E402
from lgh_b200 import problems as P  # noqa: E402


def main(argv):
    case = argv[1]
    name = argv[2] if len(argv) > 2 else "c2"
    w = int(argv[3]) if len(argv) > 3 else 220
    rtol = float(argv[4]) if len(argv) > 4 else 1e-10
    fp32 = len(argv) > 5 and argv[5] == "fp32"
    L.load()
    cfg = P.grid_problem(name)
    N = cfg["N"]
    L.kernel_timing(True)
    t0 = time.time()
    if case == "zsolve":
        Z = L.Mat(cfg["Z"])
        pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=rtol))
        X = np.random.default_rng(0).standard_normal((N, w))
        L.test_zsolve(pr, X, fp32=fp32)
        info = pr.info()
    elif case == "spmm":
        B = L.Mat(cfg["B"])
        X = np.random.default_rng(0).standard_normal((N, w))
        L.test_spmm(B, X, fp32=fp32)
        info = {}
    elif case == "build":
        B, Z = L.Mat(cfg["B"]), L.Mat(cfg["Z"])
        pr = L.Prior(Z=Z, mass=cfg["mass"], opts=L.prior_opts(ksp_rtol=rtol))
        g = L.Glr(B, pr, L.glr_opts(ell=w, seed=0, trunc_rel=0.0))
        info = g.stats()
    else:
        raise SystemExit("unknown case " + case)
    dt = time.time() - t0
    print("case %s %s w=%d: %.3f s  %s" % (case, name, w, dt, info))
    for k, (ms, n, by) in L.kernel_timing_get().items():
        if n:
            print("  %-12s launches %7d  %9.3f ms  %8.3f ms/launch  %7.1f GB/s"
                  % (k, n, ms, ms / n, by / n / (ms / n / 1e3) / 1e9))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
