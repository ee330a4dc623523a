/* api_test.cu -- kernel-level test hooks of the C ABI.
 *
 * Each hook runs exactly one device kernel path on host inputs (copied in
 * and out here) so that the parity tests can compare a single kernel with
 * the oracle: the hashed sketch, the CSR block product, the blocked
 * Z-solve, the Gram product, the Cholesky with jitter, the triangular
 * inverse and the Jacobi eigensolver.  None of them is used by the build.
 */

#include <string.h>

#include <vector>

#include "lgh_device.cuh"
#include "lgh_internal.h"
#include "lgh_mg.h"
#include "lgh_objects.h"

using namespace lgh;

template <typename T>
static int
up (DBuf<T> &d, const T *h, size_t n)
{
  LGH_TRY (d.alloc (n));
  LGH_CUDA (cudaMemcpy (d.p, h, n * sizeof (T), cudaMemcpyHostToDevice));
  return 0;
}

template <typename T>
static int
down (T *h, const DBuf<T> &d, size_t n)
{
  LGH_CUDA (cudaMemcpy (h, d.p, n * sizeof (T), cudaMemcpyDeviceToHost));
  return 0;
}

/* one Chebyshev-Jacobi step of a square CSR Mat on n x w row-major host
 * blocks (the smoother's kernel k_cheb): X is updated in place; Rout = Ro - A d_new and, with
 * CHEB_STORE_D (4) in flags, Dout = d_new.  flags as the smoother's
 * (1 first step: Do not read; 2 x is zero: X not read). */
template <typename T>
static int
test_cheb (lgh_Mat A, int w, double a, double b, int flags, double *X, const double *Ro, const double *Do, double *Rout,
           double *Dout, double bp)
{
  const int64_t n = A->csr.n;
  const int ld = round_ld (w);
  const size_t cnt = (size_t) n * ld;
  std::vector<T> hx (cnt, T (0)), hr (cnt, T (0)), hd (cnt, T (0));
  for (int64_t i = 0; i < n; i++)
    for (int j = 0; j < w; j++) {
      hx[i * ld + j] = (T) X[i * w + j];
      hr[i * ld + j] = (T) Ro[i * w + j];
      hd[i * ld + j] = Do ? (T) Do[i * w + j] : T (0);
    }
  DBuf<T> dx, dro, ddo, drn, ddn;
  LGH_TRY (up (dx, hx.data (), cnt));
  LGH_TRY (up (dro, hr.data (), cnt));
  LGH_TRY (up (ddo, hd.data (), cnt));
  LGH_TRY (drn.alloc (cnt));
  LGH_TRY (ddn.alloc (cnt));
  LGH_CUDA (cudaMemset (drn.p, 0, cnt * sizeof (T)));
  LGH_CUDA (cudaMemset (ddn.p, 0, cnt * sizeof (T)));
  LGH_TRY (launch_cheb_step<T> (A->csr, dx.p, dro.p, drn.p, ddo.p, ddn.p, ld, a, b,
                                flags, stream (), bp));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  LGH_TRY (down (hx.data (), dx, cnt));
  LGH_TRY (down (hr.data (), drn, cnt));
  LGH_TRY (down (hd.data (), ddn, cnt));
  for (int64_t i = 0; i < n; i++)
    for (int j = 0; j < w; j++) {
      X[i * w + j] = (double) hx[i * ld + j];
      Rout[i * w + j] = (double) hr[i * ld + j];
      if (Dout) Dout[i * w + j] = (double) hd[i * ld + j];
    }
  return 0;
}

extern "C" {

/* out (n x k, row-major) = Omega columns j0 .. j0+k-1 */
int
lgh_test_sketch (uint64_t seed, int64_t n, int64_t j0, int k, double *out)
{
  LGH_TRY (ensure_init ());
  const int ld = round_ld (k);
  DBuf<double> Y;
  LGH_TRY (Y.alloc ((size_t) n * ld));
  LGH_TRY (launch_sketch (seed, n, j0, k, Y.p, ld, stream ()));
  std::vector<double> h ((size_t) n * ld);
  LGH_TRY (down (h.data (), Y, h.size ()));
  for (int64_t i = 0; i < n; i++)
    memcpy (out + i * k, h.data () + i * ld, k * sizeof (double));
  return 0;
}

/* the integer xorshift states (n x k, row-major) */
int
lgh_test_rng_state (uint64_t seed, int64_t n, int64_t j0, int k, uint64_t *out)
{
  LGH_TRY (ensure_init ());
  DBuf<uint64_t> S;
  LGH_TRY (S.alloc ((size_t) n * k));
  LGH_TRY (launch_rng_state (seed, n, j0, k, S.p, stream ()));
  return down (out, S, (size_t) n * k);
}

/* Y = A X through the strip form at height R (2, 4 or 8; 0 = the cost
 * model's choice), X and Y n x w row-major; fp32 != 0 runs the float path.
 * The form is rebuilt for each call; *R_used (nullable) receives its
 * height. */
int
lgh_test_spmm_strip (lgh_Mat A, int w, const double *X, double *Y, int fp32,
                     int R, int *R_used)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (A && A->kind == 0, LGH_ERR_ARG_WRONG, "lgh_test_spmm_strip: CSR Mat");
  LGH_CHECK (R == 0 || R == 2 || R == 4 || R == 8, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_test_spmm_strip: R must be 0, 2, 4 or 8");
  StripForm S;
  LGH_TRY (strip_build (A->csr, R, S));
  if (R_used) *R_used = S.R;
  const int64_t n = A->csr.n;
  const int ld = round_ld (w);
  std::vector<double> hx ((size_t) n * ld, 0.);
  for (int64_t i = 0; i < n; i++) memcpy (hx.data () + i * ld, X + i * w, w * sizeof (double));
  std::vector<double> hy ((size_t) n * ld);
  int rc = 0;
  if (!fp32) {
    DBuf<double> dx, dy;
    if (!rc) rc = up (dx, hx.data (), hx.size ());
    if (!rc) rc = dy.alloc (hx.size ());
    if (!rc) rc = launch_strip_spmm<double> (S, dx.p, ld, dy.p, ld, w, stream ());
    if (!rc) rc = down (hy.data (), dy, hy.size ());
  } else {
    std::vector<float> fx (hx.begin (), hx.end ()), fy (hx.size ());
    DBuf<float> dx, dy;
    if (!rc) rc = up (dx, fx.data (), fx.size ());
    if (!rc) rc = dy.alloc (fx.size ());
    if (!rc) rc = launch_strip_spmm<float> (S, dx.p, ld, dy.p, ld, w, stream ());
    if (!rc) rc = down (fy.data (), dy, fy.size ());
    for (size_t e = 0; e < fy.size (); e++) hy[e] = fy[e];
  }
  strip_free (S);
  if (rc) return rc;
  for (int64_t i = 0; i < n; i++) memcpy (Y + i * w, hy.data () + i * ld, w * sizeof (double));
  return 0;
}

/* Y = A X by the row-wise CSR product, X and Y n x w row-major; fp32 != 0
 * runs the float path */
int
lgh_test_spmm (lgh_Mat A, int w, const double *X, double *Y, int fp32)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (A && A->kind == 0, LGH_ERR_ARG_WRONG, "lgh_test_spmm: CSR Mat");
  const int64_t n = A->csr.n;
  const int ld = round_ld (w);
  std::vector<double> hx ((size_t) n * ld, 0.);
  for (int64_t i = 0; i < n; i++) memcpy (hx.data () + i * ld, X + i * w, w * sizeof (double));
  std::vector<double> hy ((size_t) n * ld);
  if (!fp32) {
    DBuf<double> dx, dy;
    LGH_TRY (up (dx, hx.data (), hx.size ()));
    LGH_TRY (dy.alloc (hx.size ()));
    LGH_TRY (launch_spmm<double> (A->csr, dx.p, ld, dy.p, ld, w, stream ()));
    LGH_TRY (down (hy.data (), dy, hy.size ()));
  } else {
    std::vector<float> fx (hx.begin (), hx.end ()), fy (hx.size ());
    DBuf<float> dx, dy;
    LGH_TRY (up (dx, fx.data (), fx.size ()));
    LGH_TRY (dy.alloc (fx.size ()));
    LGH_TRY (launch_spmm<float> (A->csr, dx.p, ld, dy.p, ld, w, stream ()));
    LGH_TRY (down (fy.data (), dy, fy.size ()));
    for (size_t e = 0; e < fy.size (); e++) hy[e] = fy[e];
  }
  for (int64_t i = 0; i < n; i++) memcpy (Y + i * w, hy.data () + i * ld, w * sizeof (double));
  return 0;
}

int
lgh_test_cheb_step (lgh_Mat A, int w, double a, double b, int flags,
                    int fp32, double *X, const double *Ro,
                    const double *Do, double *Rout, double *Dout, double bp)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (A && A->kind == 0 && X && Ro && Rout, LGH_ERR_ARG_NULL,
             "lgh_test_cheb_step: NULL");
  LGH_CHECK (A->csr.ncols == 0 || A->csr.ncols == A->csr.n, LGH_ERR_ARG_WRONG,
             "lgh_test_cheb_step: square CSR Mat");
  LGH_CHECK (w >= 1, LGH_ERR_ARG_OUTOFRANGE, "lgh_test_cheb_step: w");
  return fp32 ? test_cheb<float> (A, w, a, b, flags, X, Ro, Do, Rout, Dout, bp)
              : test_cheb<double> (A, w, a, b, flags, X, Ro, Do, Rout, Dout, bp);
}

/* Y = Z^{-1} X through the prior's blocked solve, n x w row-major */
int
lgh_test_zsolve (lgh_prior_t *p, int w, const double *X, double *Y, int fp32)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (p, LGH_ERR_ARG_NULL, "lgh_test_zsolve: NULL");
  const int64_t n = p->n;
  const int ld = round_ld (w);
  std::vector<double> hx ((size_t) n * ld, 0.);
  for (int64_t i = 0; i < n; i++) memcpy (hx.data () + i * ld, X + i * w, w * sizeof (double));
  std::vector<double> hy ((size_t) n * ld);
  if (!fp32) {
    DBuf<double> dx, dy;
    LGH_TRY (up (dx, hx.data (), hx.size ()));
    LGH_TRY (dy.alloc (hx.size ()));
    LGH_TRY (prior_solve_rows<double> (p, w, dx.p, ld, nullptr, dy.p, ld, nullptr));
    LGH_TRY (down (hy.data (), dy, hy.size ()));
  } else {
    std::vector<float> fx (hx.begin (), hx.end ()), fy (hx.size ());
    DBuf<float> dx, dy;
    LGH_TRY (up (dx, fx.data (), fx.size ()));
    LGH_TRY (dy.alloc (fx.size ()));
    LGH_TRY (prior_solve_rows<float> (p, w, dx.p, ld, nullptr, dy.p, ld, nullptr));
    LGH_TRY (down (fy.data (), dy, fy.size ()));
    for (size_t e = 0; e < fy.size (); e++) hy[e] = fy[e];
  }
  for (int64_t i = 0; i < n; i++) memcpy (Y + i * w, hy.data () + i * ld, w * sizeof (double));
  return 0;
}

/* G (w x w col-major) = X^T X, X n x w row-major */
int
lgh_test_gram (int64_t n, int w, const double *X, double *G)
{
  LGH_TRY (ensure_init ());
  DBuf<double> dx, dg, work;
  LGH_TRY (up (dx, X, (size_t) n * w));
  LGH_TRY (dg.alloc ((size_t) w * w));
  LGH_TRY (work.alloc (gemm_tn_work_elems (n, w, w)));
  LGH_TRY (launch_gemm_tn<double> (n, w, w, dx.p, w, dx.p, w, dg.p, w, 0,
                                   work.p, work.n, stream ()));
  return down (G, dg, (size_t) w * w);
}

/* Y = X M, X n x k row-major, M k x m col-major */
int
lgh_test_gemm_nn (int64_t n, int k, int m, const double *X, const double *M,
                  double *Y)
{
  LGH_TRY (ensure_init ());
  DBuf<double> dx, dm, dy;
  LGH_TRY (up (dx, X, (size_t) n * k));
  LGH_TRY (up (dm, M, (size_t) k * m));
  LGH_TRY (dy.alloc ((size_t) n * m));
  LGH_TRY (launch_gemm_nn<double> (n, k, m, 1.0, dx.p, k, dm.p, k, 0.,
                                   (const double *) nullptr, 0, dy.p, m,
                                   stream ()));
  return down (Y, dy, (size_t) n * m);
}

/* lower Cholesky with the jitter retry; info[0] failed, info[1] jittered;
 * Linv (optional) = L^{-1} */
int
lgh_test_potrf (int n, const double *G, int jitter_mode, double *L,
                double *Linv, int *info)
{
  LGH_TRY (ensure_init ());
  DBuf<double> dg, d0, di;
  DBuf<int> dinf;
  LGH_TRY (up (dg, G, (size_t) n * n));
  LGH_TRY (d0.alloc ((size_t) n * n));
  LGH_TRY (dinf.alloc (4));
  LGH_TRY (launch_potrf (n, dg.p, d0.p, jitter_mode, dinf.p, stream ()));
  LGH_TRY (down (info, dinf, 2));
  LGH_TRY (down (L, dg, (size_t) n * n));
  if (Linv && !info[0]) {
    LGH_TRY (di.alloc ((size_t) n * n));
    LGH_TRY (launch_trtri_lower (n, dg.p, di.p, 0, stream ()));
    LGH_TRY (down (Linv, di, (size_t) n * n));
  }
  return 0;
}

/* Jacobi eigensolve of a symmetric n x n (col-major): w unordered, V */
int
lgh_test_syev (int n, const double *A, double *w, double *V, int *sweeps)
{
  LGH_TRY (ensure_init ());
  DBuf<double> da, da2, dv, dv2, dw;
  LGH_TRY (up (da, A, (size_t) n * n));
  LGH_TRY (da2.alloc ((size_t) n * n));
  LGH_TRY (dv.alloc ((size_t) n * n));
  LGH_TRY (dv2.alloc ((size_t) n * n));
  LGH_TRY (dw.alloc (n));
  LGH_TRY (launch_syev_jacobi (n, da.p, dv.p, dw.p, da2.p, dv2.p, sweeps,
                               stream ()));
  LGH_TRY (down (w, dw, n));
  return down (V, dv, (size_t) n * n);
}

/* the host multigrid set-up's first coarsening (no device call) */
int
lgh_test_mg_galerkin (int64_t n, const int64_t *rowptr, const int32_t *colidx,
                      const double *vals, int threads, int64_t *nc,
                      int64_t *p_rowptr, int32_t *p_colidx, double *p_vals,
                      int64_t p_cap, int64_t *p_nnz, int64_t *c_rowptr,
                      int32_t *c_colidx, double *c_vals, int64_t c_cap,
                      int64_t *c_nnz)
{
  return mg_host_galerkin (n, rowptr, colidx, vals, threads, nc, p_rowptr,
                           p_colidx, p_vals, p_cap, p_nnz, c_rowptr, c_colidx,
                           c_vals, c_cap, c_nnz);
}

} /* extern "C" */
