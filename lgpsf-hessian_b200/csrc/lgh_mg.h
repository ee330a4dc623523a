/* lgh_mg.h -- the aggregation-multigrid hierarchy (mg.cu). */

#ifndef LGH_MG_H
#define LGH_MG_H

#include <vector>

#include "lgh_internal.h"

namespace lgh
{

struct MgLevel
{
  Csr A;            /* level operator (level 0 borrows Z's arrays)      */
  Csr P, R;         /* prolongation n_l x n_{l+1}, restriction = P^T    */
  int64_t n = 0;
  double smax = 0., slo = 0., shi = 0.;
  int nu = 2;
  int own = 1;
  /* the first smoothing step of the two-step form as a plain residual
   * product r1 = r0 - F1 r0: A's pattern (F1 shares A's arrays) with the
   * values fl(b1 vd_ij) in FP64 and fl((float) b1 vd32_ij) in FP32, b1 =
   * 1 / theta, the very products the Chebyshev step forms (owned: f1v,
   * f1v32; null where the level does not smooth) */
  Csr F1;
  double *f1v = nullptr;
  float *f1v32 = nullptr;
  /* A P (n_l x n_{l+1}): the post residual after the coarse correction is
   * r2 - (A P) xc, from the pre-smoothing residual r2, without the fine
   * product A (x + P xc) (owned; empty on the coarsest level) */
  Csr AP;
};

struct MgWork
{
  int cap = 0;
  DBuf<char> B, X, R0, R1, D0, D1;
};

struct Hierarchy
{
  std::vector<MgLevel> lev;   /* 0 = finest */
  int n0 = 0;                 /* coarsest size (dense inverse)            */
  DBuf<double> Ainv;          /* n0 x n0                                  */
  std::vector<MgWork> w64, w32;
  double setup_s = 0.;
  ~Hierarchy ();
};

struct KTrace;

/* the host set-up's first coarsening of a square host CSR, on the host
 * alone (test hook; see mg.cu) */
int mg_host_galerkin (int64_t n, const int64_t *rowptr, const int32_t *colidx,
                      const double *vals, int threads, int64_t *nc_out,
                      int64_t *p_rowptr, int32_t *p_colidx, double *p_vals,
                      int64_t p_cap, int64_t *p_nnz, int64_t *c_rowptr,
                      int32_t *c_colidx, double *c_vals, int64_t c_cap,
                      int64_t *c_nnz);

/* X = V(B): one block V-cycle from the finest level (X overwritten);
 * tr (nullable) records the fine level's kernels for the timing registry;
 * work (nullable) gives the level buffers of a caller that runs V-cycles
 * beside the hierarchy's own users (the request loop), else the
 * hierarchy's shared buffers are used */
template <typename T>
int mg_vcycle (Hierarchy *h, const T *B, T *X, int ld, int w, cudaStream_t s,
               KTrace *tr = nullptr, std::vector<MgWork> *work = nullptr);

/* a Chebyshev step on a CSR operator with the Jacobi PC (zsolve.cu):
 * d_new = a d + b D^{-1} r; x += d_new; r_new = r - A d_new.  flags:
 * CHEB_FIRST (no d yet: a ignored, D not read), CHEB_ZERO_X (x is zero:
 * X not read, only written), CHEB_STORE_D (write d_new for a next step),
 * CHEB_R_ONLY (write r_new alone: neither x nor d), CHEB_PREV_R (the
 * previous step was a first step with coefficient bp run with
 * CHEB_R_ONLY: Do holds its input residual r_prev, and its d = bp D^{-1}
 * r_prev and its x are formed here with the same roundings, so the pair
 * gives the same bits as two ordinary steps) */
enum { CHEB_FIRST = 1, CHEB_ZERO_X = 2, CHEB_STORE_D = 4, CHEB_R_ONLY = 8,
       CHEB_PREV_R = 16 };
template <typename T>
int launch_cheb_step (const Csr &A, T *X, const T *Ro, T *Rn, const T *Do,
                      T *Dn, int ld, double a, double b, int flags,
                      cudaStream_t s, double bp = 0.);
/* the same step's x update alone, for a last step whose r_new is unused;
 * bp != 0: D holds the residual of a CHEB_R_ONLY first step with
 * coefficient bp (as CHEB_PREV_R above) */
template <typename T>
int launch_cheb_tail (const Csr &A, T *X, const T *R, const T *D, int ld,
                      double a, double b, int first, cudaStream_t s,
                      double bp = 0.);

int csr_finish (Csr &A);
void csr_free (Csr &A);

} /* namespace lgh */

#endif /* LGH_MG_H */
