/* correct.cu -- stage 2.5: the deflation correction against the true
 * Hessian (the reference's include/lgpsf_hessian/impl/correct_impl.h,
 * lgh_glr_correct_probes :583-800 and lgh_glr_correct :803-904).
 *
 * With S^± = (U lam U^T + c0 I)^{±1/2} and F_true = M^{1/2} Z^{-1} H_d
 * Z^{-T} M^{1/2}, the whitened error operator E_w = S^-(F_true + c0 I)S^- - I
 * is symmetric; its dominant eigenpairs (V, D) give the correction
 * F_corr = U lam U^T + Vhat D Vhat^T, Vhat = S^+ V, grafted into a new
 * (U', lam') by orthogonalisation against U and a small eigensolve
 * (correct_impl.h:325-489).  The error basis comes either from the probe
 * pairs the fit stage already has (value pass: the residuals
 * Yw - U lam U^T X of the whitened probes, no true applies) or from a hashed
 * Gaussian sketch of E_w (fresh pass); the apply budget then prices the
 * top basis directions exactly (Rayleigh values d, clamped at
 * -1 + clamp_eps, kept by |d|, signs kept).
 *
 * Every tall block is a row-major N x m device block (ld a multiple of 4),
 * as in the rest of the library: Z-solves, U passes and Gram products run
 * on the device; the true-Hessian callback gets host arrays one column at a
 * time (the reference's local arrays); the small symmetric eigenproblems
 * (m x m, m <= the apply budget or the probe count) run on the device
 * Jacobi solver.
 */

#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "lgh_internal.h"
#include "lgh_objects.h"

namespace lgh
{

namespace
{

/* Z = a X + b Y on row-major blocks (any of them may be the same) */
__global__ void
k_blk_axpby (int64_t n, int m, double a, const double *X, int ldx, double b,
             const double *Y, int ldy, double *Z, int ldz)
{
  const int64_t total = n * m;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / m;
    const int j = (int) (e - i * m);
    const double x = a != 0. ? a * X[i * ldx + j] : 0.;
    const double y = b != 0. ? b * Y[i * ldy + j] : 0.;
    Z[i * ldz + j] = x + y;
  }
}

int
ewgrid (int64_t total)
{
  int64_t g = (total + 255) / 256;
  const int64_t cap = (int64_t) num_sms () * 8;
  return (int) std::max<int64_t> (1, std::min (g, cap));
}

/* a row-major N x m device block */
struct Blk
{
  DBuf<double> d;
  int64_t n = 0;
  int m = 0, ld = 4;
  int alloc (int64_t n_, int m_)
  {
    n = n_;
    m = m_;
    ld = round_ld (std::max (m_, 1));
    LGH_TRY (d.alloc ((size_t) n * ld));
    LGH_CUDA (cudaMemsetAsync (d.p, 0, (size_t) n * ld * sizeof (double), stream ()));
    return 0;
  }
};

int
axpby (int64_t n, int m, double a, const double *X, int ldx, double b,
       const double *Y, int ldy, double *Z, int ldz)
{
  if (n == 0 || m == 0) return 0;
  k_blk_axpby<<<ewgrid (n * m), 256, 0, stream ()>>> (n, m, a, X, ldx, b, Y, ldy,
                                                      Z, ldz);
  LGH_LAUNCH_CHECK ();
  return 0;
}

/* out (host, p x q column-major) = A^T B over n rows */
int
xtY (int64_t n, const double *A, int lda, int p, const double *B, int ldb,
     int q, std::vector<double> &out)
{
  out.assign ((size_t) p * q, 0.);
  if (p == 0 || q == 0) return 0;
  DBuf<double> c, work;
  LGH_TRY (c.alloc ((size_t) p * q));
  LGH_TRY (work.alloc (std::max<size_t> (gemm_tn_work_elems (n, p, q), 64)));
  cudaStream_t s = stream ();
  LGH_TRY (launch_gemm_tn<double> (n, p, q, A, lda, B, ldb, c.p, p, 0, work.p,
                                   work.n, s));
  LGH_CUDA (cudaMemcpyAsync (out.data (), c.p, out.size () * sizeof (double),
                             cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

/* C (n x q) = alpha A (n x p) Bh + beta C, Bh host p x q column-major */
int
gemm_hb (int64_t n, double alpha, const double *A, int lda, int p,
         const std::vector<double> &Bh, int q, double beta, double *C, int ldc)
{
  if (q == 0 || n == 0) return 0;
  cudaStream_t s = stream ();
  if (p == 0) {
    if (beta != 1.) LGH_TRY (axpby (n, q, 0., C, ldc, beta, C, ldc, C, ldc));
    return 0;
  }
  DBuf<double> b;
  LGH_TRY (b.alloc ((size_t) p * q));
  LGH_CUDA (cudaMemcpyAsync (b.p, Bh.data (), (size_t) p * q * sizeof (double),
                             cudaMemcpyHostToDevice, s));
  LGH_TRY (launch_gemm_nn<double> (n, p, q, alpha, A, lda, b.p, p, beta, C, ldc,
                                   C, ldc, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

/* symmetric eigendecomposition of a small host matrix (column-major,
 * symmetric): w ascending, V column-major (the dsyevd convention) */
int
small_syev (int k, const std::vector<double> &A, std::vector<double> &w,
            std::vector<double> &V)
{
  w.assign (k, 0.);
  V.assign ((size_t) k * k, 0.);
  if (k == 0) return 0;
  cudaStream_t s = stream ();
  DBuf<double> a, a2, v, v2, wd;
  const size_t kk = (size_t) k * k;
  LGH_TRY (a.alloc (kk));
  LGH_TRY (a2.alloc (kk));
  LGH_TRY (v.alloc (kk));
  LGH_TRY (v2.alloc (kk));
  LGH_TRY (wd.alloc (k));
  LGH_CUDA (cudaMemcpyAsync (a.p, A.data (), kk * sizeof (double),
                             cudaMemcpyHostToDevice, s));
  LGH_TRY (launch_syev_jacobi (k, a.p, v.p, wd.p, a2.p, v2.p, nullptr, s));
  std::vector<double> wu (k), Vu (kk);
  LGH_CUDA (cudaMemcpyAsync (wu.data (), wd.p, k * sizeof (double),
                             cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaMemcpyAsync (Vu.data (), v.p, kk * sizeof (double),
                             cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  std::vector<int> ord (k);
  for (int i = 0; i < k; i++) ord[i] = i;
  std::stable_sort (ord.begin (), ord.end (),
                    [&] (int x, int y) { return wu[x] < wu[y]; });
  for (int j = 0; j < k; j++) {
    w[j] = wu[ord[j]];
    memcpy (&V[(size_t) j * k], &Vu[(size_t) ord[j] * k], k * sizeof (double));
  }
  return 0;
}

/* Y = f_c X + U diag(f - f_c) U^T X over m columns (f: kept values) */
int
filter_block (lgh_glr_t *g, const std::vector<double> &f, double fc,
              const double *X, int ldx, int m, double *Y, int ldy)
{
  const int64_t n = g->n;
  const int kept = g->kept;
  if (kept == 0) return axpby (n, m, fc, X, ldx, 0., X, ldx, Y, ldy);
  std::vector<double> C;
  LGH_TRY (xtY (n, g->U.p, g->ldu, kept, X, ldx, m, C));
  for (int j = 0; j < m; j++)
    for (int k = 0; k < kept; k++) C[k + (size_t) j * kept] *= f[k] - fc;
  if (Y != X) LGH_TRY (axpby (n, m, 0., X, ldx, fc, X, ldx, Y, ldy));
  else LGH_TRY (axpby (n, m, 0., X, ldx, fc, Y, ldy, Y, ldy));
  return gemm_hb (n, 1.0, g->U.p, g->ldu, kept, C, m, 1.0, Y, ldy);
}

/* Y = (U lam U^T + c I)^p X (the block form of lgh_glr_pow) */
int
pow_block (lgh_glr_t *g, double c, double p, const double *X, int ldx, int m,
           double *Y, int ldy)
{
  std::vector<double> f (g->kept);
  for (int k = 0; k < g->kept; k++) f[k] = pow (g->lam_h[k] + c, p);
  return filter_block (g, f, pow (c, p), X, ldx, m, Y, ldy);
}

/* Y = F_true X = M^{1/2} Z^{-1} H_d Z^{-T} M^{1/2} X, W scratch (n x m) */
int
ftrue_block (lgh_glr_t *g, lgh_hessian_fn hess, void *ctx, const double *X,
             int ldx, int m, double *Y, int ldy, double *W, int ldw,
             int *napplies)
{
  lgh_prior_t *p = g->prior;
  const int64_t n = g->n;
  cudaStream_t s = stream ();
  LGH_TRY (prior_solve_rows<double> (p, m, X, ldx, p->msqrt.p, Y, ldy, nullptr));
  LGH_CUDA (cudaStreamSynchronize (s));
  std::vector<double> hin (n), hout (n);
  for (int j = 0; j < m; j++) {
    LGH_CUDA (cudaMemcpy2D (hin.data (), sizeof (double), Y + j,
                            (size_t) ldy * sizeof (double), sizeof (double), n,
                            cudaMemcpyDeviceToHost));
    hess (hin.data (), hout.data (), ctx);
    LGH_CUDA (cudaMemcpy2D (W + j, (size_t) ldw * sizeof (double), hout.data (),
                            sizeof (double), sizeof (double), n,
                            cudaMemcpyHostToDevice));
  }
  *napplies += m;
  return prior_solve_rows<double> (p, m, W, ldw, nullptr, Y, ldy, p->msqrt.p);
}

/* E = E_w T = S^-((F_true + c0 I)(S^- T)) - T */
int
ew_block (lgh_glr_t *g, double c0, lgh_hessian_fn hess, void *ctx,
          const double *T, int ldt, int m, Blk &E, int *napplies)
{
  const int64_t n = g->n;
  Blk S1, S2;
  LGH_TRY (S1.alloc (n, m));
  LGH_TRY (S2.alloc (n, m));
  LGH_TRY (E.alloc (n, m));
  LGH_TRY (pow_block (g, c0, -0.5, T, ldt, m, S1.d.p, S1.ld));
  LGH_TRY (ftrue_block (g, hess, ctx, S1.d.p, S1.ld, m, S2.d.p, S2.ld, E.d.p,
                        E.ld, napplies));
  LGH_TRY (axpby (n, m, c0, S1.d.p, S1.ld, 1.0, S2.d.p, S2.ld, S2.d.p, S2.ld));
  LGH_TRY (pow_block (g, c0, -0.5, S2.d.p, S2.ld, m, E.d.p, E.ld));
  return axpby (n, m, 1.0, E.d.p, E.ld, -1.0, T, ldt, E.d.p, E.ld);
}

/* orthonormal basis of the columns of IMG, descending energy, dropping
 * directions at or below drop_tol * max(top energy, scale_floor)
 * (correct_impl.h:246-287) */
int
energy_basis (int64_t n, const double *IMG, int ldi, int k, double drop_tol,
              double scale_floor, Blk &Q, int *dim)
{
  std::vector<double> G, ev, V;
  LGH_TRY (xtY (n, IMG, ldi, k, IMG, ldi, k, G));
  LGH_TRY (small_syev (k, G, ev, V));
  const double scale = k > 0 ? std::max (ev[k - 1], scale_floor) : scale_floor;
  int nkeep = 0;
  for (int j = k - 1; j >= 0; j--) {
    if (ev[j] > drop_tol * scale && ev[j] > 0.) nkeep++;
    else break;
  }
  std::vector<double> C ((size_t) k * std::max (nkeep, 1), 0.);
  for (int j = 0; j < nkeep; j++) {
    const int idx = k - 1 - j;
    const double sc = 1. / sqrt (ev[idx]);
    for (int i = 0; i < k; i++) C[i + (size_t) j * k] = V[i + (size_t) idx * k] * sc;
  }
  LGH_TRY (Q.alloc (n, std::max (nkeep, 1)));
  if (nkeep > 0)
    LGH_TRY (gemm_hb (n, 1.0, IMG, ldi, k, C, nkeep, 0.0, Q.d.p, Q.ld));
  Q.m = nkeep;
  *dim = nkeep;
  return 0;
}

/* sqrt(|U lam U^T Xw - Yw|_F^2 / |Yw|_F^2) (correct_impl.h:290-316) */
int
qc_ratio (lgh_glr_t *g, const Blk &Xw, const Blk &Yw, double *qc)
{
  const int64_t n = g->n;
  const int m = Xw.m;
  Blk R;
  LGH_TRY (R.alloc (n, m));
  LGH_TRY (filter_block (g, g->lam_h, 0., Xw.d.p, Xw.ld, m, R.d.p, R.ld));
  LGH_TRY (axpby (n, m, 1.0, R.d.p, R.ld, -1.0, Yw.d.p, Yw.ld, R.d.p, R.ld));
  std::vector<double> gr, gy;
  LGH_TRY (xtY (n, R.d.p, R.ld, m, R.d.p, R.ld, m, gr));
  LGH_TRY (xtY (n, Yw.d.p, Yw.ld, m, Yw.d.p, Yw.ld, m, gy));
  double num = 0., den = 0.;
  for (int j = 0; j < m; j++) {
    num += gr[j + (size_t) j * m];
    den += gy[j + (size_t) j * m];
  }
  *qc = den > 0. ? sqrt (std::max (num, 0.) / den) : 0.;
  return 0;
}

/* |w|-descending order by repeated swaps (the reference's selection rule,
 * so ties resolve the same way) */
std::vector<int>
absdesc_order (const std::vector<double> &w)
{
  const int n = (int) w.size ();
  std::vector<int> o (n);
  for (int i = 0; i < n; i++) o[i] = i;
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++)
      if (fabs (w[o[j]]) > fabs (w[o[i]])) std::swap (o[i], o[j]);
  return o;
}

/* fold Vhat diag(d) Vhat^T into (U, lam) (correct_impl.h:325-489) */
int
graft (lgh_glr_t *g, const Blk &Vhat, const std::vector<double> &d, int r,
       const lgh_glr_correct_opts_t &opts, lgh_glr_correct_report_t *rep)
{
  const int64_t n = g->n;
  const int kept0 = g->kept;
  std::vector<double> Gv;
  LGH_TRY (xtY (n, Vhat.d.p, Vhat.ld, r, Vhat.d.p, Vhat.ld, r, Gv));
  double scale_floor = 0.;
  for (int i = 0; i < r; i++) scale_floor += Gv[i + (size_t) i * r];
  scale_floor /= std::max (r, 1);
  /* Vperp = (I - U U^T) Vhat */
  Blk Vperp;
  LGH_TRY (Vperp.alloc (n, r));
  LGH_TRY (axpby (n, r, 1.0, Vhat.d.p, Vhat.ld, 0., Vhat.d.p, Vhat.ld,
                  Vperp.d.p, Vperp.ld));
  std::vector<double> Cuv;
  if (kept0 > 0) {
    LGH_TRY (xtY (n, g->U.p, g->ldu, kept0, Vhat.d.p, Vhat.ld, r, Cuv));
    LGH_TRY (gemm_hb (n, -1.0, g->U.p, g->ldu, kept0, Cuv, r, 1.0, Vperp.d.p,
                      Vperp.ld));
  }
  Blk Qv;
  int r2 = 0;
  LGH_TRY (energy_basis (n, Vperp.d.p, Vperp.ld, r, opts.drop_tol, scale_floor,
                         Qv, &r2));
  std::vector<double> Cqv;
  if (r2 > 0) LGH_TRY (xtY (n, Qv.d.p, Qv.ld, r2, Vhat.d.p, Vhat.ld, r, Cqv));
  /* T2 = diag(lam, 0) + CB diag(d) CB^T on the basis [U | Qv] */
  const int n2 = kept0 + r2;
  std::vector<double> T2 ((size_t) std::max (n2, 1) * std::max (n2, 1), 0.);
  for (int i = 0; i < kept0; i++) T2[i + (size_t) i * n2] = g->lam_h[i];
  std::vector<double> CB ((size_t) std::max (n2 * r, 1), 0.);
  for (int jc = 0; jc < r; jc++) {
    for (int i = 0; i < kept0; i++) CB[i + (size_t) jc * n2] = Cuv[i + (size_t) jc * kept0];
    for (int i = 0; i < r2; i++) CB[kept0 + i + (size_t) jc * n2] = Cqv[i + (size_t) jc * r2];
  }
  for (int a = 0; a < n2; a++)
    for (int b = 0; b < n2; b++) {
      double sacc = 0.;
      for (int jc = 0; jc < r; jc++)
        sacc += CB[a + (size_t) jc * n2] * d[jc] * CB[b + (size_t) jc * n2];
      T2[a + (size_t) b * n2] += sacc;
    }
  for (int j = 0; j < n2; j++)
    for (int i = 0; i < j; i++) {
      const double avg = 0.5 * (T2[i + (size_t) j * n2] + T2[j + (size_t) i * n2]);
      T2[i + (size_t) j * n2] = avg;
      T2[j + (size_t) i * n2] = avg;
    }
  std::vector<double> ev2, V2;
  LGH_TRY (small_syev (n2, T2, ev2, V2));
  const std::vector<int> order = absdesc_order (ev2);
  const double absmax = n2 > 0 ? fabs (ev2[order[0]]) : 0.;
  double cut = 0.;
  if (g->opts.trunc_abs > 0.) cut = std::max (cut, g->opts.trunc_abs);
  if (g->opts.trunc_rel > 0.) cut = std::max (cut, g->opts.trunc_rel * absmax);
  int keptn = 0;
  while (keptn < n2 && fabs (ev2[order[keptn]]) > cut) keptn++;
  std::vector<double> lam_new (keptn);
  double lmin = 0.;
  for (int i = 0; i < keptn; i++) {
    lam_new[i] = ev2[order[i]];
    lmin = std::min (lmin, lam_new[i]);
  }
  /* U' = [U | Qv] W_sel */
  std::vector<double> Wsel ((size_t) std::max (n2, 1) * std::max (keptn, 1), 0.);
  for (int j = 0; j < keptn; j++)
    for (int i = 0; i < n2; i++)
      Wsel[i + (size_t) j * n2] = V2[i + (size_t) order[j] * n2];
  const int ldu = round_ld (std::max (keptn, 1));
  DBuf<double> Unew;
  LGH_TRY (Unew.alloc ((size_t) n * ldu));
  LGH_CUDA (cudaMemsetAsync (Unew.p, 0, (size_t) n * ldu * sizeof (double), stream ()));
  if (keptn > 0) {
    std::vector<double> Wu ((size_t) std::max (kept0, 1) * keptn, 0.);
    std::vector<double> Wq ((size_t) std::max (r2, 1) * keptn, 0.);
    for (int j = 0; j < keptn; j++) {
      for (int i = 0; i < kept0; i++) Wu[i + (size_t) j * kept0] = Wsel[i + (size_t) j * n2];
      for (int i = 0; i < r2; i++) Wq[i + (size_t) j * r2] = Wsel[kept0 + i + (size_t) j * n2];
    }
    if (kept0 > 0)
      LGH_TRY (gemm_hb (n, 1.0, g->U.p, g->ldu, kept0, Wu, keptn, 0.0, Unew.p, ldu));
    if (r2 > 0)
      LGH_TRY (gemm_hb (n, 1.0, Qv.d.p, Qv.ld, r2, Wq, keptn,
                        kept0 > 0 ? 1.0 : 0.0, Unew.p, ldu));
  }
  /* install the corrected model */
  g->U.swap (Unew);
  g->ldu = ldu;
  g->kept = keptn;
  g->lam_h = lam_new;
  LGH_TRY (g->lam_d.alloc (std::max (keptn, 1)));
  LGH_TRY (g->lraw_d.alloc (std::max (keptn, 1)));
  if (keptn > 0) {
    LGH_CUDA (cudaMemcpy (g->lam_d.p, lam_new.data (), keptn * sizeof (double),
                          cudaMemcpyHostToDevice));
    LGH_CUDA (cudaMemcpy (g->lraw_d.p, lam_new.data (), keptn * sizeof (double),
                          cudaMemcpyHostToDevice));
  }
  g->U32.release ();
  g->Wz.release ();
  g->have_wz = 0;
  g->corrected = 1;
  g->floor = std::max (0., -lmin);
  g->stats.kept = keptn;
  rep->floor = g->floor;
  return 0;
}

/* Rayleigh-price the orthonormal directions QB with their images EB,
 * clamp, keep by |d|, Vhat = S^+ (QB Vs), graft (correct_impl.h:491-580) */
int
price_and_graft (lgh_glr_t *g, const lgh_glr_correct_opts_t &opts,
                 lgh_glr_correct_report_t *rep, const Blk &QB, const Blk &EB)
{
  const int64_t n = g->n;
  const int r = QB.m;
  const double t0 = wall ();
  std::vector<double> S, ev, V;
  LGH_TRY (xtY (n, QB.d.p, QB.ld, r, EB.d.p, EB.ld, r, S));
  for (int j = 0; j < r; j++)
    for (int i = 0; i < j; i++) {
      const double avg = 0.5 * (S[i + (size_t) j * r] + S[j + (size_t) i * r]);
      S[i + (size_t) j * r] = avg;
      S[j + (size_t) i * r] = avg;
    }
  LGH_TRY (small_syev (r, S, ev, V));
  const std::vector<int> order = absdesc_order (ev);
  int rkeep = opts.rank < 0 ? r : std::min (r, opts.rank);
  while (rkeep > 0 && fabs (ev[order[rkeep - 1]]) < opts.d_keep_min) rkeep--;
  if (rkeep == 0) {
    rep->kept = 0;
    rep->clamped = 0;
    rep->d_min = r > 0 ? ev[0] : 0.;
    rep->d_max = r > 0 ? ev[r - 1] : 0.;
    rep->floor = 0.;
    return 0;
  }
  std::vector<double> dsel (rkeep), Csel ((size_t) r * rkeep);
  rep->clamped = 0;
  rep->d_min = rep->d_max = 0.;
  for (int j = 0; j < rkeep; j++) {
    double dj = ev[order[j]];
    if (dj < -1. + opts.clamp_eps) {
      dj = -1. + opts.clamp_eps;
      rep->clamped++;
    }
    dsel[j] = dj;
    rep->d_min = j == 0 ? dj : std::min (rep->d_min, dj);
    rep->d_max = j == 0 ? dj : std::max (rep->d_max, dj);
    for (int i = 0; i < r; i++) Csel[i + (size_t) j * r] = V[i + (size_t) order[j] * r];
  }
  Blk Vw, Vhat;
  LGH_TRY (Vw.alloc (n, rkeep));
  LGH_TRY (gemm_hb (n, 1.0, QB.d.p, QB.ld, r, Csel, rkeep, 0.0, Vw.d.p, Vw.ld));
  LGH_TRY (Vhat.alloc (n, rkeep));
  LGH_TRY (pow_block (g, opts.c0, 0.5, Vw.d.p, Vw.ld, rkeep, Vhat.d.p, Vhat.ld));
  LGH_TRY (graft (g, Vhat, dsel, rkeep, opts, rep));
  rep->kept = rkeep;
  rep->t_dense += wall () - t0;
  return 0;
}

/* a non-owning view of the first m columns of a block (row-major: the
 * same storage and leading dimension) */
struct View
{
  const double *p = nullptr;
  int64_t n = 0;
  int m = 0, ld = 4;
};

View
view (const Blk &b, int m)
{
  View v;
  v.p = b.d.p;
  v.n = b.n;
  v.m = m;
  v.ld = b.ld;
  return v;
}

/* [A | B] into a new block */
int
concat (const View &A, const View &B, Blk &O)
{
  LGH_TRY (O.alloc (A.n, A.m + B.m));
  cudaStream_t s = stream ();
  if (A.m > 0)
    LGH_CUDA (cudaMemcpy2DAsync (O.d.p, (size_t) O.ld * 8, A.p, (size_t) A.ld * 8,
                                 (size_t) A.m * 8, A.n, cudaMemcpyDeviceToDevice, s));
  if (B.m > 0)
    LGH_CUDA (cudaMemcpy2DAsync (O.d.p + A.m, (size_t) O.ld * 8, B.p,
                                 (size_t) B.ld * 8, (size_t) B.m * 8, A.n,
                                 cudaMemcpyDeviceToDevice, s));
  return 0;
}

/* whitened probes of host column-major (N x k) V and HV:
 * X = M^{-1/2} Z^T V (Z applies), Yw = M^{1/2} Z^{-1} HV (a block solve) */
int
whiten_probes (lgh_glr_t *g, int k, const double *Vh, const double *HVh,
               Blk &X, Blk &Yw)
{
  lgh_prior_t *p = g->prior;
  const int64_t n = g->n;
  cudaStream_t s = stream ();
  LGH_TRY (X.alloc (n, k));
  LGH_TRY (Yw.alloc (n, k));
  DBuf<double> v, y;
  LGH_TRY (v.alloc (n));
  LGH_TRY (y.alloc (n));
  for (int j = 0; j < k; j++) {
    LGH_CUDA (cudaMemcpy (v.p, Vh + (size_t) j * n, n * sizeof (double),
                          cudaMemcpyHostToDevice));
    LGH_TRY (prior_applyZ (p, v.p, y.p));
    LGH_TRY (launch_vec_div (n, y.p, p->msqrt.p, v.p, s));
    LGH_CUDA (cudaMemcpy2DAsync (X.d.p + j, (size_t) X.ld * 8, v.p, 8, 8, n,
                                 cudaMemcpyDeviceToDevice, s));
    LGH_CUDA (cudaStreamSynchronize (s));
  }
  DBuf<double> hv;
  LGH_TRY (hv.alloc ((size_t) n * k));
  LGH_CUDA (cudaMemcpy (hv.p, HVh, (size_t) n * k * sizeof (double),
                        cudaMemcpyHostToDevice));
  Blk H;
  LGH_TRY (H.alloc (n, k));
  LGH_TRY (launch_colmajor_to_rowmajor (n, k, hv.p, n, H.d.p, H.ld, nullptr, s));
  LGH_TRY (prior_solve_rows<double> (p, k, H.d.p, H.ld, nullptr, Yw.d.p, Yw.ld,
                                     p->msqrt.p));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

int
correct_checks (lgh_glr_t *glr, const lgh_glr_correct_opts_t &o, const char *who)
{
  LGH_CHECK (!glr->corrected, LGH_ERR_ORDER, "%s: the object is already corrected",
             who);
  LGH_CHECK (o.c0 > 0., LGH_ERR_ARG_OUTOFRANGE, "%s: c0 must be positive", who);
  return 0;
}

} /* namespace */

/* the corrected operator's low-rank action, y = Z M^{-1/2}(U lam U^T + c I)
 * M^{-1/2} Z v (glr.h:196-198) */
int
glr_apply_corrected (lgh_glr_t *g, double c, const double *v, double *y)
{
  lgh_prior_t *p = g->prior;
  const int64_t n = g->n;
  cudaStream_t s = stream ();
  DBuf<double> t, u;
  LGH_TRY (t.alloc (n));
  LGH_TRY (u.alloc (n));
  LGH_TRY (prior_applyZ (p, v, t.p));
  LGH_TRY (launch_vec_div (n, t.p, p->msqrt.p, u.p, s));
  std::vector<double> f (g->kept);
  for (int k = 0; k < g->kept; k++) f[k] = g->lam_h[k] + c;
  /* u (a 1-column row-major block, ld 1) */
  if (g->kept > 0) {
    std::vector<double> C;
    LGH_TRY (xtY (n, g->U.p, g->ldu, g->kept, u.p, 1, 1, C));
    for (int k = 0; k < g->kept; k++) C[k] *= f[k] - c;
    LGH_TRY (axpby (n, 1, 0., u.p, 1, c, u.p, 1, t.p, 1));
    LGH_TRY (gemm_hb (n, 1.0, g->U.p, g->ldu, g->kept, C, 1, 1.0, t.p, 1));
  } else {
    LGH_TRY (axpby (n, 1, 0., u.p, 1, c, u.p, 1, t.p, 1));
  }
  LGH_TRY (launch_vec_div (n, t.p, p->msqrt.p, u.p, s));
  LGH_TRY (prior_applyZ (p, u.p, y));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

} /* namespace lgh */

using namespace lgh;

extern "C" {

lgh_glr_correct_opts_t
lgh_glr_correct_opts_default (void)
{
  /* correct_impl.h:43-58 */
  lgh_glr_correct_opts_t o;
  o.c0 = 1.0;
  o.rank = -1;
  o.applies = 30;
  o.n_qc = 0;
  o.q_power = 0;
  o.clamp_eps = 0.05;
  o.d_keep_min = 0.;
  o.drop_tol = 1e-12;
  o.seed = 424242UL;
  o.verbose = 0;
  return o;
}

int
lgh_glr_correct_probes (lgh_glr_t *glr, int k, const double *V,
                        const double *HV, lgh_hessian_fn hess, void *ctx,
                        const lgh_glr_correct_opts_t *opts_in,
                        lgh_glr_correct_report_t *report)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (glr && V && HV && hess, LGH_ERR_ARG_NULL,
             "lgh_glr_correct_probes: NULL argument");
  const lgh_glr_correct_opts_t o = opts_in ? *opts_in : lgh_glr_correct_opts_default ();
  lgh_glr_correct_report_t rep;
  memset (&rep, 0, sizeof (rep));
  rep.qc_before = rep.qc_after = -1.;
  LGH_TRY (correct_checks (glr, o, "lgh_glr_correct_probes"));
  const int kf = k - o.n_qc;
  LGH_CHECK (kf > 0 && o.n_qc >= 0, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_correct_probes: need k - n_qc > 0 probes (k=%d, n_qc=%d)",
             k, o.n_qc);
  LGH_CHECK (o.applies > 0, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_correct_probes: applies budget must be positive");
  const int64_t n = glr->n;
  int napplies = 0;
  double t0 = wall ();
  Blk X, Yw, Xq, Yqw;
  LGH_TRY (whiten_probes (glr, kf, V, HV, X, Yw));
  rep.t_operator += wall () - t0;
  if (o.n_qc > 0) {
    LGH_TRY (whiten_probes (glr, o.n_qc, V + (size_t) kf * n, HV + (size_t) kf * n,
                            Xq, Yqw));
    LGH_TRY (qc_ratio (glr, Xq, Yqw, &rep.qc_before));
  }
  /* residual images IMG = S^-(Yw - U lam U^T X): the free error basis */
  t0 = wall ();
  Blk Rw, IMG, QB0;
  LGH_TRY (Rw.alloc (n, kf));
  LGH_TRY (filter_block (glr, glr->lam_h, 0., X.d.p, X.ld, kf, Rw.d.p, Rw.ld));
  LGH_TRY (axpby (n, kf, 1.0, Yw.d.p, Yw.ld, -1.0, Rw.d.p, Rw.ld, Rw.d.p, Rw.ld));
  LGH_TRY (IMG.alloc (n, kf));
  LGH_TRY (pow_block (glr, o.c0, -0.5, Rw.d.p, Rw.ld, kf, IMG.d.p, IMG.ld));
  int bdim = 0;
  LGH_TRY (energy_basis (n, IMG.d.p, IMG.ld, kf, o.drop_tol, 0., QB0, &bdim));
  rep.basis = bdim;
  rep.t_dense += wall () - t0;
  LGH_CHECK (bdim > 0, LGH_ERR_CONV_FAILED,
             "lgh_glr_correct_probes: the probe residuals span nothing -- either "
             "the approximation is already exact on the probes or the probe "
             "data is inconsistent");
  /* price the top m1 basis directions exactly */
  const int m1 = std::min (o.applies, bdim);
  const View Q1v = view (QB0, m1);
  Blk E1;
  t0 = wall ();
  LGH_TRY (ew_block (glr, o.c0, hess, ctx, Q1v.p, Q1v.ld, m1, E1, &napplies));
  rep.t_operator += wall () - t0;
  Blk QB, EB;
  bool have = false;
  if (o.applies > m1 && m1 > 0) {
    /* one power step past the basis */
    std::vector<double> C;
    LGH_TRY (xtY (n, Q1v.p, Q1v.ld, m1, E1.d.p, E1.ld, m1, C));
    Blk Pb;
    LGH_TRY (Pb.alloc (n, m1));
    LGH_TRY (axpby (n, m1, 1.0, E1.d.p, E1.ld, 0., E1.d.p, E1.ld, Pb.d.p, Pb.ld));
    LGH_TRY (gemm_hb (n, -1.0, Q1v.p, Q1v.ld, m1, C, m1, 1.0, Pb.d.p, Pb.ld));
    std::vector<double> Ge;
    LGH_TRY (xtY (n, E1.d.p, E1.ld, m1, E1.d.p, E1.ld, m1, Ge));
    double sf = 0.;
    for (int j = 0; j < m1; j++) sf += Ge[j + (size_t) j * m1];
    sf /= std::max (m1, 1);
    Blk Q2b;
    int b2 = 0;
    LGH_TRY (energy_basis (n, Pb.d.p, Pb.ld, m1, o.drop_tol, sf, Q2b, &b2));
    const int m2 = std::min (o.applies - m1, b2);
    if (m2 > 0) {
      const View Q2v = view (Q2b, m2);
      Blk E2;
      t0 = wall ();
      LGH_TRY (ew_block (glr, o.c0, hess, ctx, Q2v.p, Q2v.ld, m2, E2, &napplies));
      rep.t_operator += wall () - t0;
      LGH_TRY (concat (Q1v, Q2v, QB));
      LGH_TRY (concat (view (E1, m1), view (E2, m2), EB));
      have = true;
    }
  }
  if (!have) {
    LGH_TRY (concat (Q1v, View (), QB));
    LGH_TRY (concat (view (E1, m1), View (), EB));
  }
  LGH_TRY (price_and_graft (glr, o, &rep, QB, EB));
  rep.hd_applies = napplies;
  if (o.n_qc > 0) LGH_TRY (qc_ratio (glr, Xq, Yqw, &rep.qc_after));
  if (o.verbose)
    fprintf (stderr, "[lgh correct] basis %d, priced %d applies, kept %d "
             "(clamped %d), d in [%.3g, %.3g], floor %.3g, qc %.3g -> %.3g\n",
             rep.basis, rep.hd_applies, rep.kept, rep.clamped, rep.d_min,
             rep.d_max, rep.floor, rep.qc_before, rep.qc_after);
  if (report) *report = rep;
  return 0;
}

int
lgh_glr_correct (lgh_glr_t *glr, lgh_hessian_fn hess, void *ctx,
                 const lgh_glr_correct_opts_t *opts_in,
                 lgh_glr_correct_report_t *report)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (glr && hess, LGH_ERR_ARG_NULL, "lgh_glr_correct: NULL argument");
  const lgh_glr_correct_opts_t o = opts_in ? *opts_in : lgh_glr_correct_opts_default ();
  lgh_glr_correct_report_t rep;
  memset (&rep, 0, sizeof (rep));
  rep.qc_before = rep.qc_after = -1.;
  LGH_TRY (correct_checks (glr, o, "lgh_glr_correct"));
  LGH_CHECK (o.applies >= 2, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_correct: the fresh path needs applies >= 2 (range pass + "
             "Rayleigh pass)");
  const int64_t n = glr->n;
  const int passes = 2 + std::max (o.q_power, 0);
  const int mr = std::max (o.applies / passes, 1);
  int napplies = 0;
  /* hashed Gaussian test block in the whitened frame */
  Blk T, IMG;
  LGH_TRY (T.alloc (n, mr));
  LGH_TRY (launch_sketch (o.seed, n, 0, mr, T.d.p, T.ld, stream ()));
  double t0 = wall ();
  LGH_TRY (ew_block (glr, o.c0, hess, ctx, T.d.p, T.ld, mr, IMG, &napplies));
  rep.t_operator += wall () - t0;
  for (int pp = 0; pp < o.q_power; pp++) {
    Blk Tn;
    int bd = 0;
    LGH_TRY (energy_basis (n, IMG.d.p, IMG.ld, IMG.m, o.drop_tol, 0., Tn, &bd));
    if (bd == 0) break;
    t0 = wall ();
    LGH_TRY (ew_block (glr, o.c0, hess, ctx, Tn.d.p, Tn.ld, bd, IMG, &napplies));
    rep.t_operator += wall () - t0;
  }
  Blk QB0;
  int bdim = 0;
  LGH_TRY (energy_basis (n, IMG.d.p, IMG.ld, IMG.m, o.drop_tol, 0., QB0, &bdim));
  rep.basis = bdim;
  LGH_CHECK (bdim > 0, LGH_ERR_CONV_FAILED,
             "lgh_glr_correct: the error sketch spans nothing -- the "
             "approximation may already be exact");
  const int m1 = std::min (std::max (o.applies - napplies, 1), bdim);
  Blk QB, EB;
  LGH_TRY (concat (view (QB0, m1), View (), QB));
  t0 = wall ();
  LGH_TRY (ew_block (glr, o.c0, hess, ctx, QB.d.p, QB.ld, m1, EB, &napplies));
  rep.t_operator += wall () - t0;
  LGH_TRY (price_and_graft (glr, o, &rep, QB, EB));
  rep.hd_applies = napplies;
  if (report) *report = rep;
  return 0;
}

} /* extern "C" */
