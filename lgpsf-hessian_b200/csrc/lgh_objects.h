/* lgh_objects.h -- the opaque objects behind the C ABI handles. */

#ifndef LGH_OBJECTS_H
#define LGH_OBJECTS_H

#include <vector>

#include "lgh_internal.h"
#include "lgh_batch.h"
#include "lgh_strip.h"
#include "lgh_rows.h"

/* Mat: a device CSR operator (kind 0) or a dense column-block view handed
 * to blocked prior callbacks (kind 1, MATDENSE layout, not owned). */
struct lgh_mat_s
{
  int refs = 1;
  int kind = 0;
  lgh::Csr csr;
  double *data = nullptr;
  int64_t nrows = 0;
  int ncols = 0;
  int64_t ld = 0;
  /* the strip form of a CSR operator, built on its first block product
   * (k_strip.cu); strip_R: 0 = chosen by the cost model, or 2 / 4 / 8 */
  lgh::StripForm strips;
  int strips_built = 0;
  int strip_R = 0;
  /* row-sharded operator: csr holds the owned rows over local columns
   * [owned; ghosts] (csr.ncols = nloc + nghost) and rows the halo plan */
  lgh::RowsPlan *rows = nullptr;
};

/* Vec: a device vector; owns its array unless created with an array. */
struct lgh_vec_s
{
  double *d = nullptr;
  int64_t n = 0;
  int owns = 0;
};

/* struct lgh_prior (glr_common_impl.h:81-94) */
struct lgh_prior
{
  int refs = 1;
  int64_t n = 0;
  lgh::DBuf<double> mass, msqrt, minvsqrt;
  lgh::DBuf<double> tmp1, tmp2;
  /* callbacks path */
  lgh_prior_callbacks_t cb{};
  /* Mat path */
  int is_mat = 0;
  lgh_Mat Z = nullptr;
  lgh_prior_mat_opts_t mopts{};
  lgh::ZsolveCfg zcfg;
  lgh::ZWork ws64, ws32, wsv;
  int pc_type = 0;              /* LGH_PC_AMG | LGH_PC_JACOBI */
  lgh::Hierarchy *mg = nullptr; /* aggregation multigrid (AMG PC) */
  double emin = 0., emax = 0.;
  int bound_its = 0;
  lgh::ZsolveStats stats;
  long pc32_calls = 0;          /* Z-solves with the FP32 V-cycle (mixed) */
  lgh::DBuf<double> mix_in;     /* FP64 copy of an FP32 block (mixed) */
  /* row-sharded prior (Z row-sharded): the rank-local preconditioner and
   * the distributed PCG's workspace; n is the rank's row count */
  lgh::RowsPrior *rows = nullptr;
};

/* struct lgh_glr (glr_common_impl.h:252-278), device resident */
struct lgh_glr
{
  int64_t n = 0;
  lgh_Mat B = nullptr;
  lgh_prior_t *prior = nullptr;
  lgh_glr_opts_t opts{};
  lgh_exec_opts_t exec{};
  /* build product: U (n x kept, row-major, ld ldu) and the treated,
   * |lam|-descending spectrum (host mirror for lgh_glr_eigs) */
  lgh::DBuf<double> U, lam_d, lraw_d;
  lgh::DBuf<float> U32;
  int ldu = 4;
  int kept = 0;
  std::vector<double> lam_h;
  /* sketch state for the incremental extension: Q (n x ell) and the raw
   * projection A = Q^T F Q (ell x ell, column-major) */
  lgh::DBuf<double> Q, A;
  lgh::DBuf<float> Q32;
  int ldq = 4, ell = 0;
  /* deflation-correction state (correct.cu): U, lam are the corrected,
   * signed model; shifts need c > floor */
  int corrected = 0;
  double floor = 0.;
  /* scratch */
  lgh::DBuf<double> w1, w2, wk, fk, part;
  lgh::DBuf<unsigned> cnt;
  /* shift-independent precompute for the batched operations:
   * W = Z^{-1} M^{1/2} U (n x kept, row-major, ld ldu) */
  lgh::DBuf<double> Wz;
  int have_wz = 0;
  /* workspace and captured graph of the many-shift combination (batch.cu) */
  lgh::ShiftPlan *splan = nullptr;
  /* the communicator of a column-sharded build (size 0: one device) and
   * its library-owned exchange buffers */
  lgh_comm_t comm{};
  lgh::DBuf<char> xsend, xrecv;
  /* a build over row slabs: the communicator of B and the prior (null:
   * not row-sharded), the first global row and the global row count */
  const lgh_rows_comm_t *rows = nullptr;
  int64_t row0 = 0, N = 0;
  lgh_glr_stats_t stats{};
};

namespace lgh
{
void mat_release (lgh_Mat A);
int mat_mult_vec (lgh_Mat A, const double *x, double *y);
/* Y = A X for a row-major block of width w: the strip form from 8
 * columns on (built on first use), the row-wise CSR product below */
template <typename T>
int mat_mult_block (lgh_Mat A, const T *X, int ldx, T *Y, int ldy, int w,
                    cudaStream_t s);
/* build the strip form of A now if a width-w product will use it */
int mat_prepare_block (lgh_Mat A, int w);
void prior_ref (lgh_prior_t *p);
int prior_applyZ (lgh_prior_t *p, const double *x, double *y);
int prior_solve_vec (lgh_prior_t *p, const double *x, const double *s_in,
                     double *y, const double *s_out);
/* rtol_override > 0 replaces the prior's tolerance (FP32 solves of the
 * mixed build run at the execution options' inner tolerance) */
template <typename T>
int prior_solve_rows (lgh_prior_t *p, int w, const T *X, int ldx,
                      const double *s_in, T *Y, int ldy, const double *s_out,
                      double rtol_override = 0.);
int prior_solve_pc32 (lgh_prior_t *p, int w, const double *X, int ldx,
                      const double *s_in, double *Y, int ldy,
                      const double *s_out, double rtol_override = 0.);
int glr_apply_corrected (lgh_glr_t *g, double c, const double *v, double *y);
int launch_vec_div (int64_t n, const double *x, const double *d, double *y,
                    cudaStream_t s);
}

#endif /* LGH_OBJECTS_H */
