/* correct.cu -- stage 2.5: the deflation correction of a built GLR object
 * against the true data-misfit Hessian H_d (the reference's
 * include/lgpsf_hessian/impl/correct_impl.h: lgh_glr_correct_probes
 * :583-800, lgh_glr_correct :803-904, the graft :325-489).
 *
 * The mathematics.  The object holds the model U lam U^T of the whitened
 * sparse fit.  With the whitening metric S^(+-) = (U lam U^T + c0 I)^(+-1/2)
 * and the whitened true operator F_true = M^(1/2) Z^-1 H_d Z^-T M^(1/2),
 * the error of the model in that metric is the symmetric operator
 *     E_w = S^- (F_true + c0 I) S^- - I .
 * If E_w ~ V D V^T (V orthonormal, D its dominant eigenvalues, kept with
 * their signs), then F_true ~ U lam U^T + Vh D Vh^T with Vh = S^+ V, and
 * that rank-(kept + r) operator is re-diagonalised into a new (U', lam').
 * Afterwards the object serves the corrected operator at every shift above
 * floor = max(0, -min lam').
 *
 * Where the directions V come from:
 *   value pass  (lgh_glr_correct_probes): from the k probe pairs the fit
 *     stage already holds, (Omega, H_d Omega).  Whitening them costs no
 *     true applies: X = M^(-1/2) Z^T Omega satisfies F_true X = Yw with
 *     Yw = M^(1/2) Z^-1 H_d Omega, so S^-(Yw - U lam U^T X) are images of
 *     E_w (up to the S^- factor) for free; their energy-ordered basis is
 *     the search space.  The apply budget prices the leading directions
 *     exactly (one true apply each), and, budget left, one power step
 *     past them adds fresh directions.
 *   fresh pass  (lgh_glr_correct): a hashed Gaussian block in the
 *     whitened frame, pushed through E_w (plus q_power passes), then
 *     priced like the value pass.
 * Pricing: the Rayleigh quotient matrix Q^T E_w Q on the priced directions
 * Q, its eigenpairs ordered by |d|, a rank cap and a |d| floor, and a clamp
 * d >= -1 + clamp_eps (an exact error eigenvalue satisfies 1 + d > 0; the
 * clamp guards against estimation noise only).
 *
 * Design (this file).  A Deflator owns the object, the options, a device
 * workspace and the counters of one correction.  Every tall block is a
 * row-major device panel; the directions and their images are written
 * straight into column ranges of two panels sized for the whole budget, so
 * nothing is concatenated.  Every small matrix (Gram, Rayleigh, the
 * combined coefficient matrix of the re-diagonalisation) is formed on the
 * device by the split-K products or a dedicated kernel, eigendecomposed on
 * the device (cyclic Jacobi), and only its eigenvalues cross to the host,
 * where the selection rules run on a few hundred numbers; the chosen
 * eigenvector columns are gathered on the device.  The true-Hessian
 * callback receives host arrays (the reference's local arrays): a panel is
 * staged to the host as one column-major transfer, the callback runs on
 * each contiguous column, and the responses return as one transfer.
 */

#include <math.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "lgh_internal.h"
#include "lgh_objects.h"

namespace lgh
{

namespace
{

/* ---- device kernels ------------------------------------------------------ */

/* Z = a X + b Y over n rows and m columns of row-major panels (any two may
 * alias element for element) */
__global__ void
k_panel_axpby (int64_t n, int m, double a, const double *X, int ldx, double b,
               const double *Y, int ldy, double *Z, int ldz)
{
  const int64_t total = n * m;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / m;
    const int j = (int) (e - i * m);
    double v = 0.;
    if (a != 0.) v = a * X[i * ldx + j];
    if (b != 0.) v += b * Y[i * ldy + j];
    Z[i * ldz + j] = v;
  }
}

/* W (rows x cols, column-major, ld rows) : W[k, j] *= f[k] - fc */
__global__ void
k_coeff_rows (int rows, int cols, const double *f, double fc, double *W)
{
  const int64_t total = (int64_t) rows * cols;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int k = (int) (e % rows);
    W[e] *= f[k] - fc;
  }
}

/* C[:, j] = V[:, idx[j]] * s[j]  (V n x n column-major, C n x m) */
__global__ void
k_gather_cols (int n, int m, const double *V, const int *idx, const double *s,
               double *C)
{
  const int64_t total = (int64_t) n * m;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int j = (int) (e / n);
    const int i = (int) (e - (int64_t) j * n);
    C[e] = V[i + (int64_t) idx[j] * n] * s[j];
  }
}

/* the combined coefficient matrix of the re-diagonalisation on the
 * orthonormal basis [U | Qv] (n2 = kept0 + r2 columns):
 *   T2 = diag(lam, 0) + CB diag(d) CB^T,   CB (n2 x r, column-major).
 * One thread per entry pair (a <= b); both halves get the same value, so
 * T2 is exactly symmetric. */
__global__ void
k_fold_matrix (int n2, int r, int kept0, const double *CB, const double *d,
               const double *lam, double *T2)
{
  const int64_t total = (int64_t) n2 * n2;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int b = (int) (e / n2);
    const int a = (int) (e - (int64_t) b * n2);
    if (a > b) continue;
    double acc = 0.;
    for (int j = 0; j < r; j++)
      acc += CB[a + (int64_t) j * n2] * d[j] * CB[b + (int64_t) j * n2];
    if (a == b && a < kept0) acc += lam[a];
    T2[a + (int64_t) b * n2] = acc;
    T2[b + (int64_t) a * n2] = acc;
  }
}

/* partial sums of squares of a panel: part[blockIdx] = sum over the
 * block's rows of sum_j X[i, j]^2 (fixed order, then k_sum_parts) */
__global__ void __launch_bounds__ (256)
k_sumsq_part (int64_t n, int m, const double *X, int ldx, double *part)
{
  __shared__ double red[256];
  double acc = 0.;
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    for (int j = 0; j < m; j++) {
      const double x = X[i * ldx + j];
      acc += x * x;
    }
  red[threadIdx.x] = acc;
  __syncthreads ();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int) threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads ();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void
k_sum_parts (int np, const double *part, double *out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.;
    for (int i = 0; i < np; i++) s += part[i];
    *out = s;
  }
}

int
flat_grid (int64_t total)
{
  const int64_t g = (total + 255) / 256;
  return (int) std::max<int64_t> (1, std::min<int64_t> (g, (int64_t) num_sms () * 8));
}

/* ---- panels ------------------------------------------------------------- */

/* a row-major n x cols device block; column j of the panel is ptr + j with
 * the panel's leading dimension, so a column range is a sub-panel */
struct Panel
{
  DBuf<double> buf;
  int64_t n = 0;
  int cols = 0, ld = 4;
  int make (int64_t n_, int cols_)
  {
    n = n_;
    cols = cols_;
    ld = round_ld (std::max (cols_, 1));
    LGH_TRY (buf.alloc ((size_t) n * ld));
    LGH_CUDA (cudaMemsetAsync (buf.p, 0, (size_t) n * ld * sizeof (double),
                               stream ()));
    return 0;
  }
  double *at (int j) const { return buf.p + j; }
};

/* a device vector uploaded from host values */
int
upload (const std::vector<double> &h, DBuf<double> &d)
{
  LGH_TRY (d.alloc (std::max<size_t> (h.size (), 1)));
  if (!h.empty ())
    LGH_CUDA (cudaMemcpyAsync (d.p, h.data (), h.size () * sizeof (double),
                               cudaMemcpyHostToDevice, stream ()));
  return 0;
}

int
upload_idx (const std::vector<int> &h, DBuf<int> &d)
{
  LGH_TRY (d.alloc (std::max<size_t> (h.size (), 1)));
  if (!h.empty ())
    LGH_CUDA (cudaMemcpyAsync (d.p, h.data (), h.size () * sizeof (int),
                               cudaMemcpyHostToDevice, stream ()));
  return 0;
}

/* eigendecomposition of a small symmetric device matrix (column-major):
 * eigenvalues to the host, eigenvectors stay on the device, both in the
 * solver's order (index i of vals is column i of vecs) */
struct SmallEig
{
  DBuf<double> a, a2, vecs, v2, w;
  std::vector<double> vals;
  int n = 0;
  int run (int n_, const double *A)
  {
    n = n_;
    vals.assign (n, 0.);
    if (n == 0) return 0;
    const size_t nn = (size_t) n * n;
    cudaStream_t s = stream ();
    LGH_TRY (a.alloc (nn));
    LGH_TRY (a2.alloc (nn));
    LGH_TRY (vecs.alloc (nn));
    LGH_TRY (v2.alloc (nn));
    LGH_TRY (w.alloc (n));
    LGH_CUDA (cudaMemcpyAsync (a.p, A, nn * sizeof (double),
                               cudaMemcpyDeviceToDevice, s));
    LGH_TRY (launch_syev_jacobi (n, a.p, vecs.p, w.p, a2.p, v2.p, nullptr, s));
    LGH_CUDA (cudaMemcpyAsync (vals.data (), w.p, n * sizeof (double),
                               cudaMemcpyDeviceToHost, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    return 0;
  }
};

/* indices of vals ordered by decreasing |value|; equal magnitudes keep the
 * ascending order of the values (a tie has measure zero in practice) */
std::vector<int>
by_magnitude (const std::vector<double> &vals)
{
  std::vector<int> o (vals.size ());
  std::iota (o.begin (), o.end (), 0);
  std::stable_sort (o.begin (), o.end (),
                    [&] (int x, int y) { return vals[x] < vals[y]; });
  std::stable_sort (o.begin (), o.end (), [&] (int x, int y) {
    return fabs (vals[x]) > fabs (vals[y]);
  });
  return o;
}

/* ---- one correction ------------------------------------------------------- */

struct Deflator
{
  lgh_glr_t *g;
  lgh_glr_correct_opts_t o;
  lgh_hessian_fn hess;
  void *ctx;
  lgh_glr_correct_report_t *rep;
  int applies = 0;
  DBuf<double> work;      /* split-K partial sums of every small product */
  DBuf<double> small_a;   /* small products */
  DBuf<double> fdev;
  std::vector<double> hin, hout; /* host staging of the callback */
  DBuf<double> stage;     /* column-major device staging of the callback */

  int ensure_work (int m1, int m2)
  {
    return work.alloc (std::max<size_t> (gemm_tn_work_elems (g->n, m1, m2), 64));
  }

  /* C (m1 x m2, column-major, ldc) = A^T B over the object's rows */
  int product_tn (const double *A, int lda, int m1, const double *B, int ldb,
                  int m2, double *C, int ldc, int sym = 0)
  {
    if (m1 == 0 || m2 == 0) return 0;
    LGH_TRY (ensure_work (m1, m2));
    return launch_gemm_tn<double> (g->n, m1, m2, A, lda, B, ldb, C, ldc, sym,
                                   work.p, work.n, stream ());
  }

  int axpby (int m, double a, const double *X, int ldx, double b,
             const double *Y, int ldy, double *Z, int ldz)
  {
    if (m == 0 || g->n == 0) return 0;
    k_panel_axpby<<<flat_grid (g->n * m), 256, 0, stream ()>>> (
        g->n, m, a, X, ldx, b, Y, ldy, Z, ldz);
    LGH_LAUNCH_CHECK ();
    return 0;
  }

  /* Y = fc X + U diag(f - fc) U^T X on m columns: one split-K product for
   * the coefficients, a row scaling, and one product whose epilogue adds
   * fc X (Y may alias X) */
  int spectral (const std::vector<double> &f, double fc, const double *X,
                int ldx, int m, double *Y, int ldy)
  {
    const int kept = g->kept;
    if (m == 0) return 0;
    if (kept == 0) return axpby (m, fc, X, ldx, 0., X, ldx, Y, ldy);
    LGH_TRY (small_a.alloc ((size_t) kept * m));
    LGH_TRY (product_tn (g->U.p, g->ldu, kept, X, ldx, m, small_a.p, kept));
    LGH_TRY (upload (f, fdev));
    k_coeff_rows<<<flat_grid ((int64_t) kept * m), 256, 0, stream ()>>> (
        kept, m, fdev.p, fc, small_a.p);
    LGH_LAUNCH_CHECK ();
    return launch_gemm_nn<double> (g->n, kept, m, 1.0, g->U.p, g->ldu,
                                   small_a.p, kept, fc, X, ldx, Y, ldy,
                                   stream ());
  }

  /* Y = (U lam U^T + c0 I)^p X */
  int metric_pow (double p, const double *X, int ldx, int m, double *Y,
                  int ldy)
  {
    std::vector<double> f (g->kept);
    for (int k = 0; k < g->kept; k++) f[k] = pow (g->lam_h[k] + o.c0, p);
    return spectral (f, pow (o.c0, p), X, ldx, m, Y, ldy);
  }

  /* Y = F_true X (m columns), W scratch of the same shape */
  int true_whitened (const double *X, int ldx, int m, double *Y, int ldy,
                     double *W, int ldw)
  {
    lgh_prior_t *p = g->prior;
    const int64_t N = g->n;
    cudaStream_t s = stream ();
    LGH_TRY (prior_solve_rows<double> (p, m, X, ldx, p->msqrt.p, Y, ldy,
                                       nullptr));
    LGH_TRY (stage.alloc ((size_t) N * m));
    LGH_TRY (launch_rowmajor_to_colmajor (N, m, Y, ldy, stage.p, N, nullptr, s));
    hin.resize ((size_t) N * m);
    hout.resize ((size_t) N * m);
    LGH_CUDA (cudaMemcpyAsync (hin.data (), stage.p, hin.size () * sizeof (double),
                               cudaMemcpyDeviceToHost, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    for (int j = 0; j < m; j++)
      hess (hin.data () + (size_t) j * N, hout.data () + (size_t) j * N, ctx);
    applies += m;
    LGH_CUDA (cudaMemcpyAsync (stage.p, hout.data (), hout.size () * sizeof (double),
                               cudaMemcpyHostToDevice, s));
    LGH_TRY (launch_colmajor_to_rowmajor (N, m, stage.p, N, W, ldw, nullptr, s));
    return prior_solve_rows<double> (p, m, W, ldw, nullptr, Y, ldy, p->msqrt.p);
  }

  /* E = E_w T = S^-((F_true + c0 I) S^- T) - T, written into E (m columns
   * of a panel); two scratch panels of m columns */
  int error_image (const double *T, int ldt, int m, double *E, int lde)
  {
    if (m == 0) return 0;
    const double t0 = wall ();
    Panel s1, s2;
    LGH_TRY (s1.make (g->n, m));
    LGH_TRY (s2.make (g->n, m));
    LGH_TRY (metric_pow (-0.5, T, ldt, m, s1.buf.p, s1.ld));
    LGH_TRY (true_whitened (s1.buf.p, s1.ld, m, s2.buf.p, s2.ld, E, lde));
    LGH_TRY (axpby (m, o.c0, s1.buf.p, s1.ld, 1.0, s2.buf.p, s2.ld, s2.buf.p,
                    s2.ld));
    LGH_TRY (metric_pow (-0.5, s2.buf.p, s2.ld, m, E, lde));
    LGH_TRY (axpby (m, 1.0, E, lde, -1.0, T, ldt, E, lde));
    rep->t_operator += wall () - t0;
    return 0;
  }

  /* mean of the diagonal of X^T X (the mean column energy) */
  int mean_energy (const double *X, int ldx, int m, double *out)
  {
    *out = 0.;
    if (m == 0) return 0;
    const int nb = flat_grid (g->n);
    DBuf<double> part, tot;
    LGH_TRY (part.alloc (nb));
    LGH_TRY (tot.alloc (1));
    k_sumsq_part<<<nb, 256, 0, stream ()>>> (g->n, m, X, ldx, part.p);
    LGH_LAUNCH_CHECK ();
    k_sum_parts<<<1, 32, 0, stream ()>>> (nb, part.p, tot.p);
    LGH_LAUNCH_CHECK ();
    double s = 0.;
    LGH_CUDA (cudaMemcpyAsync (&s, tot.p, sizeof (double),
                               cudaMemcpyDeviceToHost, stream ()));
    LGH_CUDA (cudaStreamSynchronize (stream ()));
    *out = s / m;
    return 0;
  }

  /* An orthonormal basis of span(IMG) by decreasing energy: the Gram
   * matrix's eigenpairs (e, v) give directions IMG v / sqrt(e); directions
   * with e <= drop_tol * max(top e, floor) are dropped.  *dim = the number
   * of directions that survive; at most `limit` of them (all: limit < 0)
   * are written to the first columns of Q (ldq). */
  int energy_basis (const double *IMG, int ldi, int k, double floor_e,
                    int limit, double *Q, int ldq, int *dim)
  {
    *dim = 0;
    if (k == 0) return 0;
    DBuf<double> G;
    LGH_TRY (G.alloc ((size_t) k * k));
    LGH_TRY (product_tn (IMG, ldi, k, IMG, ldi, k, G.p, k, 1));
    SmallEig eg;
    LGH_TRY (eg.run (k, G.p));
    std::vector<int> desc (k);
    std::iota (desc.begin (), desc.end (), 0);
    std::stable_sort (desc.begin (), desc.end (),
                      [&] (int x, int y) { return eg.vals[x] > eg.vals[y]; });
    const double scale = std::max (eg.vals[desc[0]], floor_e);
    int live = 0;
    while (live < k && eg.vals[desc[live]] > 0.
           && eg.vals[desc[live]] > o.drop_tol * scale)
      live++;
    *dim = live;
    const int take = limit < 0 ? live : std::min (live, limit);
    if (take == 0 || Q == nullptr) return 0;
    std::vector<int> idx (desc.begin (), desc.begin () + take);
    std::vector<double> sc (take);
    for (int j = 0; j < take; j++) sc[j] = 1. / sqrt (eg.vals[idx[j]]);
    DBuf<int> di;
    DBuf<double> ds, C;
    LGH_TRY (upload_idx (idx, di));
    LGH_TRY (upload (sc, ds));
    LGH_TRY (C.alloc ((size_t) k * take));
    k_gather_cols<<<flat_grid ((int64_t) k * take), 256, 0, stream ()>>> (
        k, take, eg.vecs.p, di.p, ds.p, C.p);
    LGH_LAUNCH_CHECK ();
    return launch_gemm_nn<double> (g->n, k, take, 1.0, IMG, ldi, C.p, k, 0.,
                                   Q, ldq, Q, ldq, stream ());
  }

  /* sqrt(||U lam U^T Xq - Yq||_F^2 / ||Yq||_F^2) on held-out pairs */
  int holdout_ratio (const Panel &Xq, const Panel &Yq, double *out)
  {
    Panel R;
    LGH_TRY (R.make (g->n, Xq.cols));
    LGH_TRY (spectral (g->lam_h, 0., Xq.buf.p, Xq.ld, Xq.cols, R.buf.p, R.ld));
    LGH_TRY (axpby (Xq.cols, 1.0, R.buf.p, R.ld, -1.0, Yq.buf.p, Yq.ld,
                    R.buf.p, R.ld));
    double num = 0., den = 0.;
    LGH_TRY (mean_energy (R.buf.p, R.ld, R.cols, &num));
    LGH_TRY (mean_energy (Yq.buf.p, Yq.ld, Yq.cols, &den));
    *out = den > 0. ? sqrt (std::max (num, 0.) / den) : 0.;
    return 0;
  }

  /* the probe pairs (host, column-major N x k) whitened: X = M^(-1/2) Z^T V,
   * Yw = M^(1/2) Z^-1 HV */
  int whiten (int k, const double *Vh, const double *HVh, Panel &X, Panel &Yw)
  {
    lgh_prior_t *p = g->prior;
    const int64_t N = g->n;
    cudaStream_t s = stream ();
    const double t0 = wall ();
    LGH_TRY (X.make (N, k));
    LGH_TRY (Yw.make (N, k));
    DBuf<double> colv, colz;
    LGH_TRY (colv.alloc ((size_t) N * k));
    LGH_TRY (colz.alloc ((size_t) N * k));
    LGH_CUDA (cudaMemcpyAsync (colv.p, Vh, (size_t) N * k * sizeof (double),
                               cudaMemcpyHostToDevice, s));
    for (int j = 0; j < k; j++)     /* Z is symmetric: Z^T v = Z v */
      LGH_TRY (prior_applyZ (p, colv.p + (size_t) j * N, colz.p + (size_t) j * N));
    LGH_TRY (launch_colmajor_to_rowmajor (N, k, colz.p, N, X.buf.p, X.ld,
                                          p->minvsqrt.p, s));
    LGH_CUDA (cudaMemcpyAsync (colv.p, HVh, (size_t) N * k * sizeof (double),
                               cudaMemcpyHostToDevice, s));
    Panel H;
    LGH_TRY (H.make (N, k));
    LGH_TRY (launch_colmajor_to_rowmajor (N, k, colv.p, N, H.buf.p, H.ld,
                                          nullptr, s));
    LGH_TRY (prior_solve_rows<double> (p, k, H.buf.p, H.ld, nullptr, Yw.buf.p,
                                       Yw.ld, p->msqrt.p));
    LGH_CUDA (cudaStreamSynchronize (s));
    rep->t_operator += wall () - t0;
    return 0;
  }

  /* Rayleigh pricing of the r priced directions D (with their images
   * E = E_w D), then the re-diagonalisation of the corrected model */
  int price_and_fold (const Panel &D, const Panel &E, int r)
  {
    const double t0 = wall ();
    DBuf<double> S;
    LGH_TRY (S.alloc ((size_t) r * r));
    LGH_TRY (product_tn (D.buf.p, D.ld, r, E.buf.p, E.ld, r, S.p, r, 1));
    SmallEig es;
    LGH_TRY (es.run (r, S.p));
    const std::vector<int> ord = by_magnitude (es.vals);
    int keep = o.rank < 0 ? r : std::min (r, o.rank);
    while (keep > 0 && fabs (es.vals[ord[keep - 1]]) < o.d_keep_min) keep--;
    const double lo = r ? *std::min_element (es.vals.begin (), es.vals.end ()) : 0.;
    const double hi = r ? *std::max_element (es.vals.begin (), es.vals.end ()) : 0.;
    rep->clamped = 0;
    if (keep == 0) {
      /* nothing worth grafting: the object stays uncorrected */
      rep->kept = 0;
      rep->d_min = lo;
      rep->d_max = hi;
      rep->floor = 0.;
      rep->t_dense += wall () - t0;
      return 0;
    }
    std::vector<double> d (keep), unit (keep, 1.);
    std::vector<int> pick (ord.begin (), ord.begin () + keep);
    for (int j = 0; j < keep; j++) {
      d[j] = es.vals[pick[j]];
      if (d[j] < -1. + o.clamp_eps) {
        d[j] = -1. + o.clamp_eps;
        rep->clamped++;
      }
    }
    rep->d_min = *std::min_element (d.begin (), d.end ());
    rep->d_max = *std::max_element (d.begin (), d.end ());
    /* Vh = S^+ (D V_keep) */
    DBuf<int> di;
    DBuf<double> du, C;
    LGH_TRY (upload_idx (pick, di));
    LGH_TRY (upload (unit, du));
    LGH_TRY (C.alloc ((size_t) r * keep));
    k_gather_cols<<<flat_grid ((int64_t) r * keep), 256, 0, stream ()>>> (
        r, keep, es.vecs.p, di.p, du.p, C.p);
    LGH_LAUNCH_CHECK ();
    Panel Vw, Vh;
    LGH_TRY (Vw.make (g->n, keep));
    LGH_TRY (launch_gemm_nn<double> (g->n, r, keep, 1.0, D.buf.p, D.ld, C.p, r,
                                     0., Vw.buf.p, Vw.ld, Vw.buf.p, Vw.ld,
                                     stream ()));
    LGH_TRY (Vh.make (g->n, keep));
    LGH_TRY (metric_pow (0.5, Vw.buf.p, Vw.ld, keep, Vh.buf.p, Vh.ld));
    LGH_TRY (fold (Vh, d));
    rep->kept = keep;
    rep->t_dense += wall () - t0;
    return 0;
  }

  /* (U, lam) <- the eigenpairs of U lam U^T + Vh diag(d) Vh^T, kept by the
   * object's truncation rules, signed */
  int fold (const Panel &Vh, const std::vector<double> &d)
  {
    const int64_t N = g->n;
    const int r = Vh.cols;
    const int kept0 = g->kept;
    cudaStream_t s = stream ();
    /* the part of Vh outside span(U), and its energy basis Qv; the floor
     * (mean column energy of Vh) turns a correction inside span(U) into
     * r2 = 0 rather than noise columns */
    double floor_e = 0.;
    LGH_TRY (mean_energy (Vh.buf.p, Vh.ld, r, &floor_e));
    Panel Vp;
    LGH_TRY (Vp.make (N, r));
    const int n2max = kept0 + r;
    DBuf<double> CB;                  /* U^T Vh, kept0 x r */
    LGH_TRY (CB.alloc ((size_t) n2max * r));
    if (kept0 > 0) {
      LGH_TRY (product_tn (g->U.p, g->ldu, kept0, Vh.buf.p, Vh.ld, r, CB.p,
                           kept0));
      LGH_TRY (launch_gemm_nn<double> (N, kept0, r, -1.0, g->U.p, g->ldu, CB.p,
                                       kept0, 1.0, Vh.buf.p, Vh.ld, Vp.buf.p,
                                       Vp.ld, s));
    } else {
      LGH_TRY (axpby (r, 1.0, Vh.buf.p, Vh.ld, 0., Vh.buf.p, Vh.ld, Vp.buf.p,
                      Vp.ld));
    }
    Panel Qv;
    LGH_TRY (Qv.make (N, r));
    int r2 = 0;
    LGH_TRY (energy_basis (Vp.buf.p, Vp.ld, r, floor_e, -1, Qv.buf.p, Qv.ld,
                           &r2));
    const int n2 = kept0 + r2;
    /* [U^T Vh ; Qv^T Vh] with leading dimension n2 */
    DBuf<double> CBs;
    LGH_TRY (CBs.alloc ((size_t) std::max (n2, 1) * r));
    if (kept0 > 0)
      LGH_CUDA (cudaMemcpy2DAsync (CBs.p, (size_t) n2 * 8, CB.p,
                                   (size_t) kept0 * 8, (size_t) kept0 * 8, r,
                                   cudaMemcpyDeviceToDevice, s));
    if (r2 > 0)
      LGH_TRY (product_tn (Qv.buf.p, Qv.ld, r2, Vh.buf.p, Vh.ld, r,
                           CBs.p + kept0, n2));
    DBuf<double> dd, T2;
    LGH_TRY (upload (d, dd));
    LGH_TRY (T2.alloc ((size_t) std::max (n2, 1) * std::max (n2, 1)));
    k_fold_matrix<<<flat_grid ((int64_t) n2 * n2), 256, 0, s>>> (
        n2, r, kept0, CBs.p, dd.p, g->lam_d.p, T2.p);
    LGH_LAUNCH_CHECK ();
    SmallEig ef;
    LGH_TRY (ef.run (n2, T2.p));
    const std::vector<int> ord = by_magnitude (ef.vals);
    const double absmax = n2 > 0 ? fabs (ef.vals[ord[0]]) : 0.;
    double cut = 0.;
    if (g->opts.trunc_abs > 0.) cut = std::max (cut, g->opts.trunc_abs);
    if (g->opts.trunc_rel > 0.) cut = std::max (cut, g->opts.trunc_rel * absmax);
    int kn = 0;
    while (kn < n2 && fabs (ef.vals[ord[kn]]) > cut) kn++;
    std::vector<double> lam (kn), unit (std::max (kn, 1), 1.);
    double lmin = 0.;
    for (int i = 0; i < kn; i++) {
      lam[i] = ef.vals[ord[i]];
      lmin = std::min (lmin, lam[i]);
    }
    /* U' = [U | Qv] W, W = the kept eigenvectors (n2 x kn, ld n2) */
    const int ldu = round_ld (std::max (kn, 1));
    DBuf<double> Un;
    LGH_TRY (Un.alloc ((size_t) N * ldu));
    LGH_CUDA (cudaMemsetAsync (Un.p, 0, (size_t) N * ldu * sizeof (double), s));
    if (kn > 0) {
      std::vector<int> pick (ord.begin (), ord.begin () + kn);
      DBuf<int> di;
      DBuf<double> du, W;
      LGH_TRY (upload_idx (pick, di));
      LGH_TRY (upload (unit, du));
      LGH_TRY (W.alloc ((size_t) n2 * kn));
      k_gather_cols<<<flat_grid ((int64_t) n2 * kn), 256, 0, s>>> (
          n2, kn, ef.vecs.p, di.p, du.p, W.p);
      LGH_LAUNCH_CHECK ();
      if (kept0 > 0)
        LGH_TRY (launch_gemm_nn<double> (N, kept0, kn, 1.0, g->U.p, g->ldu,
                                         W.p, n2, 0., Un.p, ldu, Un.p, ldu, s));
      if (r2 > 0)
        LGH_TRY (launch_gemm_nn<double> (N, r2, kn, 1.0, Qv.buf.p, Qv.ld,
                                         W.p + kept0, n2, kept0 > 0 ? 1. : 0.,
                                         Un.p, ldu, Un.p, ldu, s));
    }
    LGH_CUDA (cudaStreamSynchronize (s));
    /* install the corrected model */
    g->U.swap (Un);
    g->ldu = ldu;
    g->kept = kn;
    g->lam_h = lam;
    LGH_TRY (g->lam_d.alloc (std::max (kn, 1)));
    LGH_TRY (g->lraw_d.alloc (std::max (kn, 1)));
    if (kn > 0) {
      LGH_CUDA (cudaMemcpy (g->lam_d.p, lam.data (), kn * sizeof (double),
                            cudaMemcpyHostToDevice));
      LGH_CUDA (cudaMemcpy (g->lraw_d.p, lam.data (), kn * sizeof (double),
                            cudaMemcpyHostToDevice));
    }
    g->U32.release ();
    g->Wz.release ();
    g->have_wz = 0;
    g->corrected = 1;
    g->floor = std::max (0., -lmin);
    g->stats.kept = kn;
    rep->floor = g->floor;
    return 0;
  }

  void trace () const
  {
    if (!o.verbose) return;
    fprintf (stderr, "lgh correction: %d basis directions, %d true applies, "
             "%d modes grafted (%d clamped), d in [%.3g, %.3g], shift floor "
             "%.3g, held-out ratio %.3g before, %.3g after\n", rep->basis,
             rep->hd_applies, rep->kept, rep->clamped, rep->d_min, rep->d_max,
             rep->floor, rep->qc_before, rep->qc_after);
  }
};

int
start (lgh_glr_t *glr, const lgh_glr_correct_opts_t *opts_in,
       lgh_glr_correct_report_t *rep, lgh_glr_correct_opts_t *o,
       const char *who)
{
  *o = opts_in ? *opts_in : lgh_glr_correct_opts_default ();
  memset (rep, 0, sizeof (*rep));
  rep->qc_before = rep->qc_after = -1.;
  LGH_CHECK (!glr->corrected, LGH_ERR_ORDER,
             "%s: this object carries a correction already (one per object)",
             who);
  LGH_CHECK (o->c0 > 0., LGH_ERR_ARG_OUTOFRANGE,
             "%s: the metric shift c0 = %g is not positive", who, o->c0);
  return 0;
}

} /* namespace */

/* y = Z M^(-1/2) (U lam U^T + c I) M^(-1/2) Z v, the corrected operator's
 * low-rank action served by lgh_glr_apply after a correction (glr.h:
 * 196-198) */
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
  Deflator dfl{};
  dfl.g = g;
  std::vector<double> f (g->kept);
  for (int k = 0; k < g->kept; k++) f[k] = g->lam_h[k] + c;
  LGH_TRY (dfl.spectral (f, c, u.p, 1, 1, t.p, 1));
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
  /* the reference's defaults (correct_impl.h:43-58) */
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
             "lgh_glr_correct_probes: the object, both probe arrays and the "
             "Hessian callback are required");
  LGH_CHECK (!glr->rows, LGH_ERR_SUP,
             "lgh_glr_correct_probes: not on a row-sharded object");
  lgh_glr_correct_report_t rep;
  Deflator dfl{};
  LGH_TRY (start (glr, opts_in, &rep, &dfl.o, "lgh_glr_correct_probes"));
  const lgh_glr_correct_opts_t &o = dfl.o;
  dfl.g = glr;
  dfl.hess = hess;
  dfl.ctx = ctx;
  dfl.rep = &rep;
  const int nfit = k - o.n_qc;
  LGH_CHECK (o.n_qc >= 0 && nfit > 0, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_correct_probes: %d probes with %d held out leaves none "
             "to build the error basis from", k, o.n_qc);
  LGH_CHECK (o.applies > 0, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_correct_probes: the true-apply budget (%d) must be at "
             "least 1", o.applies);
  const int64_t N = glr->n;
  Panel X, Yw, Xq, Yq;
  LGH_TRY (dfl.whiten (nfit, V, HV, X, Yw));
  if (o.n_qc > 0) {
    LGH_TRY (dfl.whiten (o.n_qc, V + (size_t) nfit * N, HV + (size_t) nfit * N,
                         Xq, Yq));
    LGH_TRY (dfl.holdout_ratio (Xq, Yq, &rep.qc_before));
  }
  /* the free error images S^-(Yw - U lam U^T X) */
  double t0 = wall ();
  Panel img;
  LGH_TRY (img.make (N, nfit));
  LGH_TRY (dfl.spectral (glr->lam_h, 0., X.buf.p, X.ld, nfit, img.buf.p,
                         img.ld));
  LGH_TRY (dfl.axpby (nfit, 1.0, Yw.buf.p, Yw.ld, -1.0, img.buf.p, img.ld,
                      img.buf.p, img.ld));
  LGH_TRY (dfl.metric_pow (-0.5, img.buf.p, img.ld, nfit, img.buf.p, img.ld));
  /* D will hold every priced direction and E their images: the leading
   * m1 = min(applies, basis) basis directions first, then up to
   * applies - m1 more from one power step */
  Panel D, E;
  LGH_TRY (D.make (N, o.applies));
  LGH_TRY (E.make (N, o.applies));
  int bdim = 0;
  LGH_TRY (dfl.energy_basis (img.buf.p, img.ld, nfit, 0., o.applies, D.buf.p,
                             D.ld, &bdim));
  rep.basis = bdim;
  rep.t_dense += wall () - t0;
  LGH_CHECK (bdim > 0, LGH_ERR_CONV_FAILED,
             "lgh_glr_correct_probes: the whitened probe residuals are all "
             "zero to rounding, so there is no error direction to correct "
             "(the model already reproduces the probes, or HV does not "
             "match V)");
  const int m1 = std::min (o.applies, bdim);
  LGH_TRY (dfl.error_image (D.buf.p, D.ld, m1, E.buf.p, E.ld));
  int priced = m1;
  if (o.applies > m1) {
    /* the images' components outside the priced directions, and their
     * energy basis (floored by the images' mean energy) */
    Panel P;
    LGH_TRY (P.make (N, m1));
    DBuf<double> Cm;
    LGH_TRY (Cm.alloc ((size_t) m1 * m1));
    LGH_TRY (dfl.product_tn (D.buf.p, D.ld, m1, E.buf.p, E.ld, m1, Cm.p, m1));
    LGH_TRY (launch_gemm_nn<double> (N, m1, m1, -1.0, D.buf.p, D.ld, Cm.p, m1,
                                     1.0, E.buf.p, E.ld, P.buf.p, P.ld,
                                     stream ()));
    double fe = 0.;
    LGH_TRY (dfl.mean_energy (E.buf.p, E.ld, m1, &fe));
    int b2 = 0;
    const int want = o.applies - m1;
    LGH_TRY (dfl.energy_basis (P.buf.p, P.ld, m1, fe, want, D.at (m1), D.ld,
                               &b2));
    const int m2 = std::min (want, b2);
    if (m2 > 0) {
      LGH_TRY (dfl.error_image (D.at (m1), D.ld, m2, E.at (m1), E.ld));
      priced += m2;
    }
  }
  D.cols = E.cols = priced;
  LGH_TRY (dfl.price_and_fold (D, E, priced));
  rep.hd_applies = dfl.applies;
  if (o.n_qc > 0) LGH_TRY (dfl.holdout_ratio (Xq, Yq, &rep.qc_after));
  dfl.trace ();
  if (report) *report = rep;
  return 0;
}

int
lgh_glr_correct (lgh_glr_t *glr, lgh_hessian_fn hess, void *ctx,
                 const lgh_glr_correct_opts_t *opts_in,
                 lgh_glr_correct_report_t *report)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (glr && hess, LGH_ERR_ARG_NULL,
             "lgh_glr_correct: the object and the Hessian callback are "
             "required");
  LGH_CHECK (!glr->rows, LGH_ERR_SUP,
             "lgh_glr_correct: not on a row-sharded object");
  lgh_glr_correct_report_t rep;
  Deflator dfl{};
  LGH_TRY (start (glr, opts_in, &rep, &dfl.o, "lgh_glr_correct"));
  const lgh_glr_correct_opts_t &o = dfl.o;
  dfl.g = glr;
  dfl.hess = hess;
  dfl.ctx = ctx;
  dfl.rep = &rep;
  LGH_CHECK (o.applies >= 2, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_correct: a budget of %d true applies cannot pay for "
             "both the range pass and the pricing pass (need >= 2)",
             o.applies);
  const int64_t N = glr->n;
  /* the budget splits over the range pass, q_power power passes and the
   * pricing pass */
  const int width = std::max (o.applies / (2 + std::max (o.q_power, 0)), 1);
  Panel T, img;
  LGH_TRY (T.make (N, width));
  LGH_TRY (img.make (N, width));
  LGH_TRY (launch_sketch (o.seed, N, 0, width, T.buf.p, T.ld, stream ()));
  LGH_TRY (dfl.error_image (T.buf.p, T.ld, width, img.buf.p, img.ld));
  int cols = width;
  for (int pass = 0; pass < o.q_power; pass++) {
    int bd = 0;
    LGH_TRY (dfl.energy_basis (img.buf.p, img.ld, cols, 0., -1, T.buf.p, T.ld,
                               &bd));
    if (bd == 0) break;
    cols = bd;
    LGH_TRY (dfl.error_image (T.buf.p, T.ld, cols, img.buf.p, img.ld));
  }
  /* what is left of the budget prices the leading directions */
  const int left = std::max (o.applies - dfl.applies, 1);
  Panel D, E;
  LGH_TRY (D.make (N, left));
  LGH_TRY (E.make (N, left));
  int bdim = 0;
  LGH_TRY (dfl.energy_basis (img.buf.p, img.ld, cols, 0., left, D.buf.p, D.ld,
                             &bdim));
  rep.basis = bdim;
  LGH_CHECK (bdim > 0, LGH_ERR_CONV_FAILED,
             "lgh_glr_correct: the sketched error images are all zero to "
             "rounding, so there is no error direction to correct (the model "
             "may already be exact)");
  const int m1 = std::min (left, bdim);
  LGH_TRY (dfl.error_image (D.buf.p, D.ld, m1, E.buf.p, E.ld));
  LGH_TRY (dfl.price_and_fold (D, E, m1));
  rep.hd_applies = dfl.applies;
  dfl.trace ();
  if (report) *report = rep;
  return 0;
}

} /* extern "C" */
