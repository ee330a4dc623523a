"""TEST INFRASTRUCTURE ONLY: ctypes binding of the parity oracle.

The oracle (``lgh_oracle.cpp``) is a plain FP64 CPU restatement of
NickAlger/lgpsf-hessian's GLR replicated backend and its downstream
operations (include/lgpsf_hessian/impl/glr_common_impl.h,
glr_scalapack_impl.h:689-915 for the incremental extension,
zsolve_impl.h for the Z-solve semantics).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
this module, and only as the checker or the timed CPU baseline; the product
library never loads it.

``ref_pure()`` loads the reference's own PETSc-free functions
(lgh_randn_at, lgh_zs_cheb_count) compiled from the reference tree by
``build_ref.sh``; it exists only where that tree was present at build time.
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

c_dbl_p = ctypes.POINTER(ctypes.c_double)


class GlrOpts(ctypes.Structure):
    """Field-for-field lgh_glr_opts_t (include/lgpsf_hessian/glr.h:68-86)."""

    _fields_ = [
        ("ell", ctypes.c_int),
        ("q_power", ctypes.c_int),
        ("trunc_abs", ctypes.c_double),
        ("trunc_rel", ctypes.c_double),
        ("treat", ctypes.c_int),
        ("seed", ctypes.c_ulong),
        ("backend", ctypes.c_int),
        ("nb", ctypes.c_int),
        ("panel", ctypes.c_int),
        ("grid2d", ctypes.c_int),
        ("check", ctypes.c_int),
    ]


class GlrReport(ctypes.Structure):
    """lgh_glr_report_t (include/lgpsf_hessian/glr.h:90-102)."""

    _fields_ = [
        ("kept", ctypes.c_int),
        ("lam_abs_max", ctypes.c_double),
        ("lam_raw_min", ctypes.c_double),
        ("lam_raw_max", ctypes.c_double),
        ("next_abs", ctypes.c_double),
        ("n_negative_raw", ctypes.c_int),
        ("resid_max", ctypes.c_double),
        ("t_operator", ctypes.c_double),
        ("t_dense", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def opts_default(**kw):
    """lgh_glr_opts_default (glr_common_impl.h:295-312) with overrides."""
    o = GlrOpts(ell=200, q_power=1, trunc_abs=0.0, trunc_rel=1e-3, treat=0,
                seed=271828, backend=0, nb=64, panel=64, grid2d=0, check=1)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liblgh_oracle.so")
    if not os.path.exists(path):
        raise RuntimeError("oracle not built: run make -C oracle")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    I64 = ctypes.c_int64
    L.orc_randn_at.restype = ctypes.c_double
    L.orc_randn_at.argtypes = [ctypes.c_uint64, I64, I64]
    L.orc_rng_state_at.restype = ctypes.c_uint64
    L.orc_rng_state_at.argtypes = [ctypes.c_uint64, I64, I64]
    L.orc_sketch.argtypes = [ctypes.c_uint64, I64, I64, ctypes.c_int, c_dbl_p]
    L.orc_csr_create.restype = P
    L.orc_csr_create.argtypes = [I64, P, P, P]
    L.orc_csr_destroy.argtypes = [P]
    L.orc_csr_mult.argtypes = [P, c_dbl_p, c_dbl_p]
    L.orc_dsyevd.restype = ctypes.c_int
    L.orc_dsyevd.argtypes = [ctypes.c_int, c_dbl_p, c_dbl_p, ctypes.c_int]
    L.orc_set_threads.argtypes = [ctypes.c_int]
    L.orc_cheb_count.restype = ctypes.c_int
    L.orc_cheb_count.argtypes = [ctypes.c_double] * 3
    L.orc_prior_create.restype = P
    L.orc_prior_create.argtypes = [I64, P, P, P, P, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int]
    L.orc_prior_info.argtypes = [P, c_dbl_p]
    L.orc_prior_destroy.argtypes = [P]
    L.orc_prior_solveZ.restype = ctypes.c_int
    L.orc_prior_solveZ.argtypes = [P, c_dbl_p, c_dbl_p]
    L.orc_prior_applyZ.argtypes = [P, c_dbl_p, c_dbl_p]
    L.orc_prior_apply.argtypes = [P, c_dbl_p, c_dbl_p]
    L.orc_prior_solve_block.argtypes = [P, ctypes.c_int, c_dbl_p, c_dbl_p]
    L.orc_glr_compute.restype = ctypes.c_int
    L.orc_glr_compute.argtypes = [P, P, ctypes.POINTER(GlrOpts), ctypes.c_int,
                                  ctypes.POINTER(P), ctypes.POINTER(GlrReport)]
    L.orc_glr_extend.restype = ctypes.c_int
    L.orc_glr_extend.argtypes = [P, ctypes.c_int, ctypes.POINTER(GlrReport)]
    L.orc_glr_destroy.argtypes = [P]
    L.orc_glr_eigs.restype = ctypes.c_int
    L.orc_glr_eigs.argtypes = [P, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(c_dbl_p)]
    L.orc_glr_U.restype = c_dbl_p
    L.orc_glr_U.argtypes = [P]
    for nm in ("orc_glr_solve", "orc_glr_sample", "orc_glr_apply"):
        f = getattr(L, nm)
        f.restype = ctypes.c_int
        f.argtypes = [P, ctypes.c_double, c_dbl_p, c_dbl_p]
    L.orc_glr_factor.restype = ctypes.c_int
    L.orc_glr_factor.argtypes = [P, ctypes.c_double, ctypes.c_int, c_dbl_p,
                                 c_dbl_p]
    L.orc_glr_pow.restype = ctypes.c_int
    L.orc_glr_pow.argtypes = [P, ctypes.c_double, ctypes.c_double, c_dbl_p,
                              c_dbl_p]
    L.orc_glr_filter.restype = ctypes.c_int
    L.orc_glr_filter.argtypes = [P, c_dbl_p, ctypes.c_double, c_dbl_p,
                                 c_dbl_p]
    L.orc_glr_filter_block.argtypes = [P, c_dbl_p, ctypes.c_double,
                                       ctypes.c_int, c_dbl_p, c_dbl_p]
    L.orc_glr_logdet.restype = ctypes.c_double
    L.orc_glr_logdet.argtypes = [P, ctypes.c_double]
    L.orc_glr_apply_F.argtypes = [P, ctypes.c_int, c_dbl_p, c_dbl_p]
    L.orc_glr_context.restype = P
    L.orc_glr_context.argtypes = [P, P]
    L.orc_cholqr2.restype = ctypes.c_int
    L.orc_cholqr2.argtypes = [I64, ctypes.c_int, c_dbl_p]
    L.orc_glr_compute_cap.restype = ctypes.c_int
    L.orc_glr_compute_cap.argtypes = [P, P, ctypes.POINTER(GlrOpts),
                                      ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(P),
                                      ctypes.POINTER(GlrReport)]
    L.orc_build_begin.restype = P
    L.orc_build_begin.argtypes = [P, P, ctypes.POINTER(GlrOpts), ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int]
    L.orc_build_step.restype = ctypes.c_int
    L.orc_build_step.argtypes = [P]
    L.orc_build_finish.restype = P
    L.orc_build_finish.argtypes = [P, ctypes.POINTER(GlrReport)]
    L.orc_glr_solve_block.restype = ctypes.c_int
    L.orc_glr_solve_block.argtypes = [P, ctypes.c_double, ctypes.c_int,
                                      c_dbl_p, c_dbl_p]
    _LIB = L
    return L


def _dp(a):
    return a.ctypes.data_as(c_dbl_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ref_pure():
    """The reference's own lgh_randn_at / lgh_zs_cheb_count, or None."""
    path = os.path.join(_HERE, "_ref", "liblgh_ref_pure.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.ref_randn_at.restype = ctypes.c_double
    L.ref_randn_at.argtypes = [ctypes.c_ulong, ctypes.c_long, ctypes.c_long]
    L.ref_cheb_count.restype = ctypes.c_long
    L.ref_cheb_count.argtypes = [ctypes.c_double] * 3
    return L


def set_threads(n=0):
    """OpenMP and OpenBLAS threads of the oracle (0: every host core)."""
    lib().orc_set_threads(int(n) if n and n > 0 else (os.cpu_count() or 1))


def randn_at(seed, i, j):
    return lib().orc_randn_at(seed, i, j)


def sketch(seed, n, j0, k):
    """Omega columns j0..j0+k-1, returned row-major (n, k)."""
    out = np.empty((k, n), dtype=np.float64)
    lib().orc_sketch(seed, n, j0, k, _dp(out))
    return out.T.copy()


class Csr:
    """Host CSR handle inside the oracle."""

    def __init__(self, rowptr, colidx, vals):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        self.vals = _f64(vals)
        self.n = len(self.rowptr) - 1
        self.h = lib().orc_csr_create(self.n, self.rowptr.ctypes.data,
                                      self.colidx.ctypes.data,
                                      self.vals.ctypes.data)

    def mult(self, x):
        x = _f64(x)
        y = np.empty_like(x)
        lib().orc_csr_mult(self.h, _dp(x), _dp(y))
        return y

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_csr_destroy(self.h)
            self.h = None


class Prior:
    """Mat-path prior (lgh_prior_create_mat): Z as CSR + lumped mass."""

    def __init__(self, Z, mass, ksp_rtol=1e-12, mode=0, tile=64,
                 cheb_rtol=1e-10, bound_maxit=200, pc="jacobi"):
        """pc: "jacobi" (default) or "amg" (the oracle's own smoothed-
        aggregation V-cycle, the stand-in for the reference's PCGAMG)."""
        self.Z = Z
        self.mass = _f64(mass)
        self.h = lib().orc_prior_create(Z.n, Z.rowptr.ctypes.data,
                                        Z.colidx.ctypes.data,
                                        Z.vals.ctypes.data,
                                        self.mass.ctypes.data, ksp_rtol,
                                        mode, tile, cheb_rtol, bound_maxit,
                                        1 if pc == "amg" else 0)
        self.n = Z.n

    def info(self):
        out = np.zeros(7)
        lib().orc_prior_info(self.h, _dp(out))
        return dict(emin=out[0], emax=out[1], lmin=out[2], lmax=out[3],
                    nit=int(out[4]), bound_its=int(out[5]),
                    mean_cg_its=out[6])

    def solveZ(self, b):
        b = _f64(b)
        x = np.empty_like(b)
        its = lib().orc_prior_solveZ(self.h, _dp(b), _dp(x))
        return x, its

    def applyZ(self, x):
        x = _f64(x)
        y = np.empty_like(x)
        lib().orc_prior_applyZ(self.h, _dp(x), _dp(y))
        return y

    def apply(self, x):
        x = _f64(x)
        y = np.empty_like(x)
        lib().orc_prior_apply(self.h, _dp(x), _dp(y))
        return y

    def solve_block(self, X):
        """X row-major (n, m) -> Z^{-1} X, row-major (n, m)."""
        Xc = _f64(np.asarray(X).T)
        Y = np.empty_like(Xc)
        lib().orc_prior_solve_block(self.h, Xc.shape[0], _dp(Xc), _dp(Y))
        return Y.T.copy()

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_prior_destroy(self.h)
            self.h = None


class Glr:
    """Oracle GLR object (lgh_glr_compute and the downstream operations)."""

    def __init__(self, B, prior, opts=None, incremental=True, cap=0,
                 _handle=None, _report=None):
        self.B = B
        self.prior = prior
        self.opts = opts if opts is not None else opts_default()
        self.n = B.n
        if _handle is not None:          # handed over by Build.finish
            self.h = _handle
            self.report = _report
            return
        self.h = ctypes.c_void_p()
        rep = GlrReport()
        rc = lib().orc_glr_compute_cap(B.h, prior.h, ctypes.byref(self.opts),
                                       1 if incremental else 0, int(cap),
                                       ctypes.byref(self.h),
                                       ctypes.byref(rep))
        if rc != 0:
            raise RuntimeError("orc_glr_compute failed: %d" % rc)
        self.report = rep.as_dict()

    def extend(self, k):
        rep = GlrReport()
        rc = lib().orc_glr_extend(self.h, k, ctypes.byref(rep))
        if rc != 0:
            raise RuntimeError("orc_glr_extend failed: %d" % rc)
        self.report = rep.as_dict()
        return self.report

    def eigs(self):
        nk = ctypes.c_int()
        p = c_dbl_p()
        lib().orc_glr_eigs(self.h, ctypes.byref(nk), ctypes.byref(p))
        return np.ctypeslib.as_array(p, shape=(max(nk.value, 1),))[
            :nk.value].copy()

    def U(self):
        k = len(self.eigs())
        p = lib().orc_glr_U(self.h)
        return np.ctypeslib.as_array(p, shape=(max(k, 1) * self.n,))[
            :k * self.n].reshape(k, self.n).T.copy()

    def _vv(self, fn, c, v):
        v = _f64(v)
        out = np.empty_like(v)
        rc = fn(self.h, c, _dp(v), _dp(out))
        if rc != 0:
            raise RuntimeError("oracle op failed: %d" % rc)
        return out

    def solve(self, c, rhs):
        return self._vv(lib().orc_glr_solve, c, rhs)

    def solve_block(self, c, R):
        """lgh_glr_solve on the columns of R (n x m), column-parallel."""
        Rf = np.asfortranarray(R, dtype=np.float64)
        X = np.empty_like(Rf)
        rc = lib().orc_glr_solve_block(self.h, c, Rf.shape[1], _dp(Rf),
                                       _dp(X))
        if rc != 0:
            raise RuntimeError("oracle solve_block failed: %d" % rc)
        return X

    def sample(self, c, xi):
        return self._vv(lib().orc_glr_sample, c, xi)

    def apply(self, c, v):
        return self._vv(lib().orc_glr_apply, c, v)

    def factor(self, c, which, v):
        v = _f64(v)
        out = np.empty_like(v)
        rc = lib().orc_glr_factor(self.h, c, which, _dp(v), _dp(out))
        if rc != 0:
            raise RuntimeError("oracle factor failed: %d" % rc)
        return out

    def pow(self, c, p, v):
        v = _f64(v)
        out = np.empty_like(v)
        rc = lib().orc_glr_pow(self.h, c, p, _dp(v), _dp(out))
        if rc != 0:
            raise RuntimeError("oracle pow failed: %d" % rc)
        return out

    def filter(self, f_lam, f_c, v):
        v = _f64(v)
        f = _f64(f_lam)
        out = np.empty_like(v)
        lib().orc_glr_filter(self.h, _dp(f), f_c, _dp(v), _dp(out))
        return out

    def logdet(self, c):
        return lib().orc_glr_logdet(self.h, c)

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None and self.h.value:
            _LIB.orc_glr_destroy(self.h)
            self.h = ctypes.c_void_p()


class Build:
    """The oracle's replicated build advanced one bounded piece at a time
    (one sketch, one wave of `wave` F-apply columns, one CholQR2, the
    Rayleigh-Ritz step, one wave of the residual check).  Stepping to the
    end gives the same object, bit for bit, as Glr(...) on the same
    arguments."""

    def __init__(self, B, prior, opts, cap=0, wave=0, incremental=True):
        self.B, self.prior, self.opts = B, prior, opts
        self.h = lib().orc_build_begin(B.h, prior.h, ctypes.byref(opts),
                                       1 if incremental else 0, int(cap),
                                       int(wave))
        if not self.h:
            raise RuntimeError("orc_build_begin: bad ell")
        self.done = False

    def step(self):
        """Run one piece; True while pieces remain."""
        st = lib().orc_build_step(self.h)
        if st < 0:
            raise RuntimeError("oracle build step failed: %d" % -st)
        self.done = st == 0
        return not self.done

    def finish(self):
        rep = GlrReport()
        h = lib().orc_build_finish(self.h, ctypes.byref(rep))
        self.h = None
        if not h:
            raise RuntimeError("oracle build not finished")
        return Glr(self.B, self.prior, self.opts, _handle=ctypes.c_void_p(h),
                   _report=rep.as_dict())

    def __del__(self):
        # an unfinished build (abandoned part way) releases its object
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_build_finish(self.h, None)
            self.h = None


def build_pieces(ell, q_power, kept, wave, check=True):
    """Number of Build.step() calls of a build whose kept count is `kept`
    (sketch, (q_power + 2) F-applies in waves, q_power + 1 CholQR2, the
    Rayleigh-Ritz step, the check's waves)."""
    w = wave if wave > 0 else ell
    n = 1 + (q_power + 2) * (-(-ell // w)) + (q_power + 1) + 1
    if check and kept > 0:
        n += -(-kept // w)
    return n


def dsyevd(A, vecs=False):
    """LAPACK dsyevd of a symmetric matrix: (w ascending, V or None)."""
    n = A.shape[0]
    a = np.array(A, dtype=np.float64, order="F")
    w = np.empty(n)
    info = lib().orc_dsyevd(n, a.ctypes.data_as(c_dbl_p), _dp(w),
                            1 if vecs else 0)
    if info != 0:
        raise RuntimeError("dsyevd info=%d" % info)
    return w, (a if vecs else None)
