/* lgh_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the parity oracle.
 *
 * A plain C++ (FP64, CPU) restatement of NickAlger/lgpsf-hessian's GLR
 * replicated backend and its downstream operations, used by the tests, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * It is never linked into, loaded by, or called from the product library
 * (lgpsf-hessian_b200/liblgh_b200.so); the product has no CPU fallback.
 *
 * Every routine cites the reference file:line it restates (paths are
 * relative to the reference project root).  Dense BLAS/LAPACK comes from the
 * OpenBLAS bundled in the scipy wheel (symbols scipy_dgemm_ etc.), the same
 * LP64 Fortran interface the reference binds in
 * include/lgpsf_hessian/impl/f77_decls.h:16-55.
 *
 * Deliberate deviations from the reference (PETSc is absent here):
 *   - Z-solves: the reference's default per-column KSP is CG + PCGAMG
 *     (zsolve_impl.h:808-818).  GAMG is replaced by a smoothed-aggregation
 *     V-cycle written here (or, on request, by Jacobi); the CG recurrence,
 *     the preconditioned-norm stopping test at ksp_rtol and the 10000-
 *     iteration cap follow PETSc's KSPCG defaults.  Blocked mode 2 runs the
 *     reference's Chebyshev core (zsolve_impl.h:108-141) with the Jacobi
 *     preconditioner, bounds from CG-Lanczos on the reference's
 *     deterministic probe (zsolve_impl.h:737-764).
 *   - MPI: one rank; every MPI_Allreduce is the identity.
 *
 * Parity pins: the RNG is checked bit-for-bit against the reference's own
 * lgh_randn_at compiled from its source (oracle/build_ref.sh), and the
 * build/ops against the dense-LAPACK gates of tests/test_glr.cpp and
 * tests/test_prior_mat.cpp (tests/test_oracle_*.py).
 */

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
void scipy_dgemm_ (const char *, const char *, const int *, const int *,
                   const int *, const double *, const double *, const int *,
                   const double *, const int *, const double *, double *,
                   const int *);
void scipy_dgemv_ (const char *, const int *, const int *, const double *,
                   const double *, const int *, const double *, const int *,
                   const double *, double *, const int *);
void scipy_dtrsm_ (const char *, const char *, const char *, const char *,
                   const int *, const int *, const double *, const double *,
                   const int *, double *, const int *);
void scipy_dsyevd_ (const char *, const char *, const int *, double *,
                    const int *, double *, double *, const int *, int *,
                    const int *, int *);
void scipy_dpotrf_ (const char *, const int *, double *, const int *, int *);
void scipy_openblas_set_num_threads (int);
}

static double
now_s ()
{
  return std::chrono::duration<double> (
             std::chrono::steady_clock::now ().time_since_epoch ())
      .count ();
}

/* ================================================================== */
/* hashed Gaussian kit: glr_common_impl.h:32-73                         */

typedef struct
{
  uint64_t s;
  int have;
  double spare;
} orc_rng_t;

/* xorshift64* + polar Box-Muller (glr_common_impl.h:35-53) */
static double
orc_randn (orc_rng_t *r)
{
  if (r->have) { r->have = 0; return r->spare; }
  for (;;) {
    uint64_t x;
    double u1, u2, s;
    x = r->s; x ^= x >> 12; x ^= x << 25; x ^= x >> 27; r->s = x;
    u1 = (double) ((x * 2685821657736338717ULL) >> 11) / 9007199254740992.0;
    x = r->s; x ^= x >> 12; x ^= x << 25; x ^= x >> 27; r->s = x;
    u2 = (double) ((x * 2685821657736338717ULL) >> 11) / 9007199254740992.0;
    u1 = 2. * u1 - 1.; u2 = 2. * u2 - 1.; s = u1 * u1 + u2 * u2;
    if (s > 0. && s < 1.) {
      double f = sqrt (-2. * log (s) / s);
      r->spare = u2 * f; r->have = 1;
      return u1 * f;
    }
  }
}

/* splitmix64 of (seed, i, j) -> nonzero state -> one draw
 * (glr_common_impl.h:59-73) */
extern "C" double
orc_randn_at (uint64_t seed, int64_t i, int64_t j)
{
  orc_rng_t r;
  uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t) (i + 1)
               + 0xC2B2AE3D27D4EB4FULL * (uint64_t) (j + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  r.s = z ? z : 0x853C49E6748FEA9BULL;
  r.have = 0;
  return orc_randn (&r);
}

/* the initial xorshift state for (seed, i, j): the integer-only part,
 * exposed so tests can check it bit-exactly against the device kernel.  */
extern "C" uint64_t
orc_rng_state_at (uint64_t seed, int64_t i, int64_t j)
{
  uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t) (i + 1)
               + 0xC2B2AE3D27D4EB4FULL * (uint64_t) (j + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return z ? z : 0x853C49E6748FEA9BULL;
}

/* Omega block, column-major n x k, columns j0..j0+k-1
 * (glr_common_impl.h:435-445; glr_scalapack_impl.h:726-729) */
extern "C" void
orc_sketch (uint64_t seed, int64_t n, int64_t j0, int k, double *out)
{
#pragma omp parallel for schedule(static)
  for (int j = 0; j < k; j++)
    for (int64_t i = 0; i < n; i++)
      out[i + (size_t) j * n] = orc_randn_at (seed, i, j0 + j);
}

/* ================================================================== */
/* CSR matrices (stand-in for PETSc AIJ; only MatMult is ever called)   */

struct orc_csr
{
  int64_t n;
  std::vector<int64_t> rowptr;
  std::vector<int> colidx;
  std::vector<double> vals;
};

static void
csr_mult (const orc_csr *A, const double *x, double *y)
{
  for (int64_t i = 0; i < A->n; i++) {
    double s = 0.;
    for (int64_t k = A->rowptr[i]; k < A->rowptr[i + 1]; k++)
      s += A->vals[k] * x[A->colidx[k]];
    y[i] = s;
  }
}

static void
csr_mult_par (const orc_csr *A, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A->n; i++) {
    double s = 0.;
    for (int64_t k = A->rowptr[i]; k < A->rowptr[i + 1]; k++)
      s += A->vals[k] * x[A->colidx[k]];
    y[i] = s;
  }
}

extern "C" orc_csr *
orc_csr_create (int64_t n, const int64_t *rowptr, const int *colidx,
                const double *vals)
{
  orc_csr *A = new orc_csr;
  A->n = n;
  A->rowptr.assign (rowptr, rowptr + n + 1);
  A->colidx.assign (colidx, colidx + rowptr[n]);
  A->vals.assign (vals, vals + rowptr[n]);
  return A;
}

extern "C" void
orc_csr_destroy (orc_csr *A)
{
  delete A;
}

extern "C" void
orc_csr_mult (const orc_csr *A, const double *x, double *y)
{
  csr_mult_par (A, x, y);
}

/* ================================================================== */
/* small LAPACK helpers                                                 */

/* eigenvalues (ascending) and, if vecs, eigenvectors in place of A
 * (LAPACK dsyevd "V"/"N", "U": glr_common_impl.h:496-514) */
extern "C" int
orc_dsyevd (int n, double *A, double *w, int vecs)
{
  int lwork = -1, liwork = -1, iwkopt = 0, info = 0;
  double wkopt;
  const char *jobz = vecs ? "V" : "N";
  scipy_dsyevd_ (jobz, "U", &n, A, &n, w, &wkopt, &lwork, &iwkopt, &liwork,
                 &info);
  lwork = (int) wkopt; liwork = iwkopt;
  std::vector<double> work ((size_t) std::max (lwork, 1));
  std::vector<int> iwork ((size_t) std::max (liwork, 1));
  scipy_dsyevd_ (jobz, "U", &n, A, &n, w, work.data (), &lwork, iwork.data (),
                 &liwork, &info);
  return info;
}

extern "C" void
orc_set_threads (int nt)
{
  scipy_openblas_set_num_threads (nt);
#ifdef _OPENMP
  omp_set_num_threads (nt);
#endif
}

/* ================================================================== */
/* aggregation multigrid for the oracle's CG: the stand-in for the
 * reference's PCGAMG (zsolve_impl.h:808-818).  Smoothed aggregation with
 * the constant near-null space, Galerkin coarse operators, Chebyshev-
 * Jacobi smoothing (nu = 2 on [0.1, 1.1] lambda_max(D^{-1}A)), dense
 * Cholesky on the coarsest level (LAPACK).  One V-cycle per CG
 * iteration.                                                            */

extern "C" {
void scipy_dpotrs_ (const char *, const int *, const int *, const double *,
                    const int *, double *, const int *, int *);
}

struct orc_mglev
{
  orc_csr A, P, R; /* R = P^T */
  std::vector<double> dinv;
  double lmax;
};

struct orc_mg
{
  std::vector<orc_mglev> lev;
  int n0 = 0;
  std::vector<double> chol; /* coarse Cholesky factor, column-major */
};

static void
csr_transpose (const orc_csr &A, int64_t ncols, orc_csr &T)
{
  T.n = ncols;
  T.rowptr.assign (ncols + 1, 0);
  for (int64_t k = 0; k < A.rowptr[A.n]; k++) T.rowptr[A.colidx[k] + 1]++;
  for (int64_t i = 0; i < ncols; i++) T.rowptr[i + 1] += T.rowptr[i];
  T.colidx.resize (A.rowptr[A.n]);
  T.vals.resize (A.rowptr[A.n]);
  std::vector<int64_t> pos (T.rowptr.begin (), T.rowptr.end () - 1);
  for (int64_t i = 0; i < A.n; i++)
    for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++) {
      int64_t p = pos[A.colidx[k]]++;
      T.colidx[p] = (int) i;
      T.vals[p] = A.vals[k];
    }
}

static void
csr_product (const orc_csr &A, const orc_csr &B, int64_t bcols, orc_csr &C)
{
  C.n = A.n;
  C.rowptr.assign (A.n + 1, 0);
  C.colidx.clear ();
  C.vals.clear ();
  std::vector<double> acc (bcols, 0.);
  std::vector<int64_t> mark (bcols, -1);
  std::vector<int> cols;
  for (int64_t i = 0; i < A.n; i++) {
    cols.clear ();
    for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++) {
      const int j = A.colidx[k];
      for (int64_t q = B.rowptr[j]; q < B.rowptr[j + 1]; q++) {
        const int c = B.colidx[q];
        if (mark[c] != i) { mark[c] = i; acc[c] = 0.; cols.push_back (c); }
        acc[c] += A.vals[k] * B.vals[q];
      }
    }
    std::sort (cols.begin (), cols.end ());
    for (int c : cols) { C.colidx.push_back (c); C.vals.push_back (acc[c]); }
    C.rowptr[i + 1] = (int64_t) C.colidx.size ();
  }
}

/* lambda_max(D^{-1} A) by 30 power iterations from a hashed start */
static double
power_lmax (const orc_csr &A, const std::vector<double> &dinv)
{
  const int64_t n = A.n;
  std::vector<double> v (n), w (n);
  for (int64_t i = 0; i < n; i++) v[i] = 0.5 + orc_randn_at (20260813ULL, i, 0);
  double nrm = 1.;
  for (int it = 0; it < 30; it++) {
    csr_mult (&A, v.data (), w.data ());
    double s = 0.;
    for (int64_t i = 0; i < n; i++) { w[i] *= dinv[i]; s += w[i] * w[i]; }
    nrm = sqrt (s);
    for (int64_t i = 0; i < n; i++) v[i] = w[i] / nrm;
  }
  return nrm;
}

static orc_mg *
orc_mg_build (const orc_csr &Z)
{
  orc_mg *h = new orc_mg;
  orc_csr A = Z;
  for (int l = 0; l < 12; l++) {
    orc_mglev lv;
    lv.A = A;
    lv.dinv.assign (A.n, 0.);
    for (int64_t i = 0; i < A.n; i++)
      for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++)
        if (A.colidx[k] == i) lv.dinv[i] = 1. / A.vals[k];
    lv.lmax = power_lmax (A, lv.dinv) * 1.05;
    if (A.n <= 1500 || l == 11) {
      const int n0 = (int) A.n;
      h->n0 = n0;
      h->chol.assign ((size_t) n0 * n0, 0.);
      for (int64_t i = 0; i < A.n; i++)
        for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++)
          h->chol[i + (size_t) A.colidx[k] * n0] = A.vals[k];
      int info = 0;
      scipy_dpotrf_ ("L", &n0, h->chol.data (), &n0, &info);
      h->lev.push_back (lv);
      break;
    }
    /* greedy aggregation over all off-diagonal couplings */
    const int64_t n = A.n;
    std::vector<int64_t> agg (n, -1);
    int64_t nc = 0;
    for (int64_t i = 0; i < n; i++) {
      if (agg[i] >= 0) continue;
      bool ok = true;
      for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++)
        if (A.colidx[k] != i && agg[A.colidx[k]] >= 0) { ok = false; break; }
      if (!ok) continue;
      agg[i] = nc;
      for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++) agg[A.colidx[k]] = nc;
      nc++;
    }
    std::vector<int64_t> a1 = agg;
    for (int64_t i = 0; i < n; i++) {
      if (a1[i] >= 0) continue;
      double best = -1.;
      for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++) {
        const int j = A.colidx[k];
        if (j != i && a1[j] >= 0 && fabs (A.vals[k]) > best) {
          best = fabs (A.vals[k]);
          agg[i] = a1[j];
        }
      }
    }
    for (int64_t i = 0; i < n; i++)
      if (agg[i] < 0) agg[i] = nc++;
    std::vector<double> sz (nc, 0.), p0 (n);
    for (int64_t i = 0; i < n; i++) sz[agg[i]] += 1.;
    for (int64_t i = 0; i < n; i++) p0[i] = 1. / sqrt (sz[agg[i]]);
    /* smoothed prolongator P = (I - omega D^{-1} A) P0 */
    const double omega = (4. / 3.) / (lv.lmax / 1.05);
    orc_csr P;
    P.n = n;
    P.rowptr.assign (n + 1, 0);
    std::vector<int64_t> cols;
    std::vector<double> vals;
    for (int64_t i = 0; i < n; i++) {
      cols.clear ();
      vals.clear ();
      auto add = [&] (int64_t c, double v) {
        for (size_t t = 0; t < cols.size (); t++)
          if (cols[t] == c) { vals[t] += v; return; }
        cols.push_back (c);
        vals.push_back (v);
      };
      add (agg[i], p0[i]);
      for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; k++)
        add (agg[A.colidx[k]], -omega * lv.dinv[i] * A.vals[k] * p0[A.colidx[k]]);
      std::vector<size_t> ord (cols.size ());
      for (size_t t = 0; t < ord.size (); t++) ord[t] = t;
      std::sort (ord.begin (), ord.end (),
                 [&] (size_t a, size_t b) { return cols[a] < cols[b]; });
      for (size_t t : ord)
        if (vals[t] != 0.) { P.colidx.push_back ((int) cols[t]); P.vals.push_back (vals[t]); }
      P.rowptr[i + 1] = (int64_t) P.colidx.size ();
    }
    orc_csr R, AP, Ac;
    csr_transpose (P, nc, R);
    csr_product (A, P, nc, AP);
    csr_product (R, AP, nc, Ac);
    lv.P = P;
    lv.R = R;
    h->lev.push_back (lv);
    A = Ac;
  }
  return h;
}

/* Chebyshev-Jacobi smoothing, correction form (zsolve_impl.h:386-404) */
static void
orc_mg_smooth (const orc_mglev &lv, const double *b, double *x)
{
  const int64_t n = lv.A.n;
  const double lo = 0.1 * lv.lmax, hi = 1.1 * lv.lmax / 1.05;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
  const double sigma1 = theta / delta;
  double rho_old = 1. / sigma1;
  std::vector<double> r (n), d (n), ad (n);
  csr_mult (&lv.A, x, ad.data ());
  for (int64_t i = 0; i < n; i++) r[i] = b[i] - ad[i];
  for (int k = 1; k <= 2; k++) {
    if (k == 1) {
      for (int64_t i = 0; i < n; i++) d[i] = lv.dinv[i] * r[i] / theta;
    } else {
      const double rho = 1. / (2. * sigma1 - rho_old);
      for (int64_t i = 0; i < n; i++)
        d[i] = rho * rho_old * d[i] + 2. * rho / delta * lv.dinv[i] * r[i];
      rho_old = rho;
    }
    for (int64_t i = 0; i < n; i++) x[i] += d[i];
    csr_mult (&lv.A, d.data (), ad.data ());
    for (int64_t i = 0; i < n; i++) r[i] -= ad[i];
  }
}

static void
orc_mg_vcycle (const orc_mg *h, size_t l, const double *b, double *x)
{
  const orc_mglev &lv = h->lev[l];
  const int64_t n = lv.A.n;
  if (l + 1 == h->lev.size ()) {
    int n0 = h->n0, one = 1, info = 0;
    for (int64_t i = 0; i < n; i++) x[i] = b[i];
    scipy_dpotrs_ ("L", &n0, &one, h->chol.data (), &n0, x, &n0, &info);
    return;
  }
  for (int64_t i = 0; i < n; i++) x[i] = 0.;
  orc_mg_smooth (lv, b, x);
  std::vector<double> r (n), bc (lv.R.n), xc (lv.R.n);
  csr_mult (&lv.A, x, r.data ());
  for (int64_t i = 0; i < n; i++) r[i] = b[i] - r[i];
  csr_mult (&lv.R, r.data (), bc.data ());
  orc_mg_vcycle (h, l + 1, bc.data (), xc.data ());
  csr_mult (&lv.P, xc.data (), r.data ());
  for (int64_t i = 0; i < n; i++) x[i] += r[i];
  orc_mg_smooth (lv, b, x);
}

/* ================================================================== */
/* the prior: glr_common_impl.h:81-244 and zsolve_impl.h:93-141,720-823 */

struct orc_prior
{
  int refs;
  int64_t n;
  std::vector<double> mass, msqrt, minvsqrt, dinv;
  orc_csr Z;
  /* lgh_prior_mat_opts_t fields used on this path (prior.h:76-89) */
  double ksp_rtol;
  int mode, tile;
  double cheb_rtol;
  int ksp_maxit;
  /* mode-2 Chebyshev state (zsolve_impl.h:74-76) */
  double lmin, lmax, emin, emax;
  int nit, bound_its;
  /* counters */
  long cg_its_total, cg_solves;
  orc_mg *mg; /* aggregation multigrid preconditioner, or NULL (Jacobi) */
};

/* PCG on one column, Jacobi preconditioner: PETSc KSPCG (Hestenes-Stiefel
 * form) with KSP_NORM_PRECONDITIONED and KSPConvergedDefault at rtol,
 * zero initial guess (zsolve_impl.h:674-683, 808-818).  If alpha/beta are
 * non-NULL the CG coefficients are recorded for the Lanczos bound estimate
 * (KSPComputeExtremeSingularValues, zsolve_impl.h:178-196).  Returns its. */
static int
pcg_column (const orc_prior *p, const double *b, double *x, double rtol,
            int maxit, std::vector<double> *alph, std::vector<double> *bet)
{
  const int64_t n = p->n;
  std::vector<double> r (b, b + n), z (n), pp (n), w (n);
  double beta = 0., betaold = 1., dp, rnorm0;
  auto pc = [&] () {
    if (p->mg) orc_mg_vcycle (p->mg, 0, r.data (), z.data ());
    else for (int64_t i = 0; i < n; i++) z[i] = p->dinv[i] * r[i];
  };
  for (int64_t i = 0; i < n; i++) x[i] = 0.;
  pc ();
  dp = 0.;
  for (int64_t i = 0; i < n; i++) dp += z[i] * z[i];
  dp = sqrt (dp);
  rnorm0 = dp;
  if (rnorm0 == 0.) return 0;
  int it;
  for (it = 0; it < maxit; it++) {
    beta = 0.;
    for (int64_t i = 0; i < n; i++) beta += r[i] * z[i];
    if (it == 0) {
      for (int64_t i = 0; i < n; i++) pp[i] = z[i];
    } else {
      double bb = beta / betaold;
      if (bet) bet->push_back (bb);
      for (int64_t i = 0; i < n; i++) pp[i] = z[i] + bb * pp[i];
    }
    betaold = beta;
    csr_mult (&p->Z, pp.data (), w.data ());
    double dpi = 0.;
    for (int64_t i = 0; i < n; i++) dpi += pp[i] * w[i];
    double a = beta / dpi;
    if (alph) alph->push_back (a);
    for (int64_t i = 0; i < n; i++) {
      x[i] += a * pp[i];
      r[i] -= a * w[i];
    }
    pc ();
    dp = 0.;
    for (int64_t i = 0; i < n; i++) dp += z[i] * z[i];
    dp = sqrt (dp);
    if (dp <= rtol * rnorm0) { it++; break; }
  }
  return it;
}

/* extreme eigenvalues of the Lanczos tridiagonal built from CG
 * coefficients: T(k,k) = 1/a_k + b_{k-1}/a_{k-1}, T(k,k+1) =
 * sqrt(b_k)/a_k (the construction behind KSPComputeExtremeSingularValues
 * for CG). */
static void
lanczos_extremes (const std::vector<double> &a, const std::vector<double> &b,
                  double *emin, double *emax)
{
  const int m = (int) a.size ();
  std::vector<double> T ((size_t) m * m, 0.), w (m);
  for (int k = 0; k < m; k++) {
    double d = 1. / a[k];
    if (k > 0) d += b[k - 1] / a[k - 1];
    T[k + (size_t) k * m] = d;
    if (k + 1 < m) {
      double e = sqrt (b[k]) / a[k];
      T[k + (size_t) (k + 1) * m] = e;
      T[k + 1 + (size_t) k * m] = e;
    }
  }
  orc_dsyevd (m, T.data (), w.data (), 0);
  *emin = w[0];
  *emax = w[m - 1];
}

/* iteration count (zsolve_impl.h:94-102) */
extern "C" int
orc_cheb_count (double lmin, double lmax, double tol)
{
  const double kap = lmax / lmin;
  const double rho = (sqrt (kap) - 1.) / (sqrt (kap) + 1.);
  return (int) ceil (log (2. / tol) / log (1. / rho));
}

/* Chebyshev core on one column block (zsolve_impl.h:108-141) with the
 * Jacobi row-scale PC (zsolve_impl.h:144-152).  X = 0, R = B on entry. */
static void
cheb_core_col (const orc_prior *p, double lmin, double lmax, int nit,
               double *X, double *R)
{
  const int64_t n = p->n;
  const double theta = 0.5 * (lmax + lmin);
  const double delta = 0.5 * (lmax - lmin);
  const double sigma1 = theta / delta;
  double rho_old = 1.0 / sigma1, rho;
  std::vector<double> Zb (n), D (n), AD (n);
  for (int64_t i = 0; i < n; i++) Zb[i] = p->dinv[i] * R[i];
  for (int64_t i = 0; i < n; i++) D[i] = Zb[i] / theta;
  for (int64_t i = 0; i < n; i++) X[i] += D[i];
  csr_mult (&p->Z, D.data (), AD.data ());
  for (int64_t i = 0; i < n; i++) R[i] -= AD[i];
  for (int k = 2; k <= nit; k++) {
    for (int64_t i = 0; i < n; i++) Zb[i] = p->dinv[i] * R[i];
    rho = 1.0 / (2.0 * sigma1 - rho_old);
    for (int64_t i = 0; i < n; i++)
      D[i] = rho * rho_old * D[i] + 2.0 * rho / delta * Zb[i];
    for (int64_t i = 0; i < n; i++) X[i] += D[i];
    csr_mult (&p->Z, D.data (), AD.data ());
    for (int64_t i = 0; i < n; i++) R[i] -= AD[i];
    rho_old = rho;
  }
}

/* lgh_prior_mat_opts_default (glr_common_impl.h:99-112) + the create path
 * (zsolve_impl.h:720-823).  mode 0: per-column CG; mode 2: blocked
 * Chebyshev with bounds from a CG-Lanczos probe solve (probe rhs
 * randn_at(0xB0BD5, i, 0), rtol 1e-12, bound_maxit its; widened by 0.9 /
 * 1.1, zsolve_impl.h:737-764). */
extern "C" orc_prior *
orc_prior_create (int64_t n, const int64_t *zrowptr, const int *zcol,
                  const double *zval, const double *mass, double ksp_rtol,
                  int mode, int tile, double cheb_rtol, int bound_maxit,
                  int use_mg)
{
  orc_prior *p = new orc_prior;
  p->refs = 1;
  p->n = n;
  p->mass.assign (mass, mass + n);
  p->msqrt.resize (n);
  p->minvsqrt.resize (n);
  for (int64_t i = 0; i < n; i++) {
    p->msqrt[i] = sqrt (fabs (mass[i]));       /* VecSqrtAbs  */
    p->minvsqrt[i] = 1. / p->msqrt[i];        /* VecReciprocal */
  }
  p->Z.n = n;
  p->Z.rowptr.assign (zrowptr, zrowptr + n + 1);
  p->Z.colidx.assign (zcol, zcol + zrowptr[n]);
  p->Z.vals.assign (zval, zval + zrowptr[n]);
  p->dinv.assign (n, 0.);
  for (int64_t i = 0; i < n; i++)
    for (int64_t k = zrowptr[i]; k < zrowptr[i + 1]; k++)
      if (zcol[k] == i) p->dinv[i] = 1. / zval[k];
  p->ksp_rtol = ksp_rtol;
  p->ksp_maxit = 10000;
  p->mode = mode;
  p->tile = tile;
  p->cheb_rtol = cheb_rtol;
  p->lmin = p->lmax = p->emin = p->emax = 0.;
  p->nit = 0;
  p->bound_its = 0;
  p->cg_its_total = 0;
  p->cg_solves = 0;
  p->mg = use_mg ? orc_mg_build (p->Z) : NULL;
  if (mode >= 2) {
    std::vector<double> rhs (n), y (n), al, be;
    for (int64_t i = 0; i < n; i++) rhs[i] = orc_randn_at (0xB0BD5ULL, i, 0);
    p->bound_its = pcg_column (p, rhs.data (), y.data (), 1e-12, bound_maxit,
                               &al, &be);
    lanczos_extremes (al, be, &p->emin, &p->emax);
    p->lmin = 0.9 * p->emin;
    p->lmax = 1.1 * p->emax;
    p->nit = orc_cheb_count (p->lmin, p->lmax, cheb_rtol);
  }
  return p;
}

extern "C" void
orc_prior_info (const orc_prior *p, double *out)
{
  out[0] = p->emin; out[1] = p->emax; out[2] = p->lmin; out[3] = p->lmax;
  out[4] = p->nit; out[5] = p->bound_its;
  out[6] = p->cg_solves ? (double) p->cg_its_total / p->cg_solves : 0.;
}

static void
prior_ref (orc_prior *p) { p->refs++; }

extern "C" void
orc_prior_destroy (orc_prior *p)
{
  if (p == NULL || --p->refs > 0) return;
  delete p->mg;
  delete p;
}

/* single-vector solve: always the KSP path (prior.h:73-75) */
extern "C" int
orc_prior_solveZ (orc_prior *p, const double *b, double *x)
{
  int its = pcg_column (p, b, x, p->ksp_rtol, p->ksp_maxit, NULL, NULL);
  p->cg_its_total += its; p->cg_solves++;
  return its;
}

extern "C" void
orc_prior_applyZ (const orc_prior *p, const double *x, double *y)
{
  csr_mult_par (&p->Z, x, y);
}

/* blocked solve, column-major n x m (lgh_prior_solve_block,
 * glr_common_impl.h:205-234 -> lgh_prior_mat_solveZ_blocked,
 * zsolve_impl.h:686-715; mode 2 tiles: lgh_zs_blocked_asolve,
 * zsolve_impl.h:600-644).  Columns are independent in both modes, so the
 * tile loop is restated column by column (a zero-padded tile column does
 * not change the others). */
extern "C" void
orc_prior_solve_block (orc_prior *p, int m, const double *X, double *Y)
{
  const int64_t n = p->n;
  long its = 0;
  if (p->mode >= 2) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < m; j++) {
      std::vector<double> R (X + (size_t) j * n, X + (size_t) (j + 1) * n);
      double *Yj = Y + (size_t) j * n;
      for (int64_t i = 0; i < n; i++) Yj[i] = 0.;
      cheb_core_col (p, p->lmin, p->lmax, p->nit, Yj, R.data ());
    }
    return;
  }
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : its)
  for (int j = 0; j < m; j++)
    its += pcg_column (p, X + (size_t) j * n, Y + (size_t) j * n,
                       p->ksp_rtol, p->ksp_maxit, NULL, NULL);
  p->cg_its_total += its;
  p->cg_solves += m;
}

/* y = R x = Z M^{-1} Z x (glr_common_impl.h:236-244) */
extern "C" void
orc_prior_apply (const orc_prior *p, const double *x, double *y)
{
  std::vector<double> w (p->n);
  csr_mult_par (&p->Z, x, w.data ());
  for (int64_t i = 0; i < p->n; i++) w[i] /= p->mass[i];
  csr_mult_par (&p->Z, w.data (), y);
}

/* ================================================================== */
/* the GLR object: glr_common_impl.h:252-278                             */

typedef struct
{
  int ell, q_power;
  double trunc_abs, trunc_rel;
  int treat;
  unsigned long seed;
  int backend, nb, panel, grid2d, check;
} orc_glr_opts_t; /* field-for-field lgh_glr_opts_t (glr.h:68-86) */

typedef struct
{
  int kept;
  double lam_abs_max, lam_raw_min, lam_raw_max, next_abs;
  int n_negative_raw;
  double resid_max, t_operator, t_dense;
} orc_glr_report_t; /* lgh_glr_report_t (glr.h:90-102) */

struct orc_glr
{
  int64_t n;
  const orc_csr *B;
  orc_prior *prior;
  orc_glr_opts_t opts;
  int incremental; /* extend: 0 = replicated rebuild, 1 = incremental */
  std::vector<double> U;   /* n x kept, column-major */
  std::vector<double> lam; /* treated, |lam|-descending */
  int kept;
  int cap; /* keep at most cap modes (rank r + oversample p: ell = r + p,
            * cap = r); 0 = no cap.  An extension of this build, not a
            * reference option; the device library applies the same rule. */
  /* sketch state kept for the incremental extension: Q (n x ell) and the
   * raw projected A = Q^T F Q (ell x ell, column-major) */
  std::vector<double> Q, A;
};

/* Y = F X (glr_common_impl.h:316-336), column-major n x m */
static void
apply_F_block (orc_glr *g, int m, const double *X, double *Y)
{
  const int64_t n = g->n;
  std::vector<double> W ((size_t) n * m);
  for (int j = 0; j < m; j++)
    for (int64_t i = 0; i < n; i++)
      W[i + (size_t) j * n] = X[i + (size_t) j * n] * g->prior->msqrt[i];
  orc_prior_solve_block (g->prior, m, W.data (), Y);    /* Z^{-T}: symmetric */
#pragma omp parallel for schedule(dynamic, 1)
  for (int j = 0; j < m; j++)
    csr_mult (g->B, Y + (size_t) j * n, W.data () + (size_t) j * n);
  orc_prior_solve_block (g->prior, m, W.data (), Y);
  for (int j = 0; j < m; j++)
    for (int64_t i = 0; i < n; i++) Y[i + (size_t) j * n] *= g->prior->msqrt[i];
}

/* G = X^T X (glr_common_impl.h:340-366) */
static void
gram (int64_t n, int ncols, const double *X, double *G)
{
  int bm = (int) n, bn = ncols;
  double one = 1.0, zero = 0.0;
  scipy_dgemm_ ("T", "N", &bn, &bn, &bm, &one, X, &bm, X, &bm, &zero, G, &bn);
}

/* CholQR2 with one diagonal jitter retry (glr_common_impl.h:370-407).
 * Returns 0, or 76 (PETSC_ERR_LIB) when potrf fails twice. */
static int
cholqr2 (int64_t n, int ncols, double *X)
{
  std::vector<double> G ((size_t) ncols * ncols);
  for (int pass = 0; pass < 2; pass++) {
    int bn = ncols, info = 0;
    gram (n, ncols, X, G.data ());
    for (int attempt = 0; attempt < 2; attempt++) {
      scipy_dpotrf_ ("L", &bn, G.data (), &bn, &info);
      if (info == 0) break;
      gram (n, ncols, X, G.data ());
      double tr = 0.;
      for (int i = 0; i < ncols; i++) tr += G[i + (size_t) i * ncols];
      for (int i = 0; i < ncols; i++) G[i + (size_t) i * ncols] += 1e-12 * tr / ncols;
    }
    if (info != 0) return 76;
    int sm = (int) n, sn = ncols;
    double one = 1.0;
    scipy_dtrsm_ ("R", "L", "T", "N", &sm, &sn, &one, G.data (), &sn, X, &sm);
  }
  return 0;
}

/* panel CholQR2 with the distributed backend's jitter rule
 * (glr_scalapack_impl.h:110-148) */
static int
panel_cholqr (double *pa, int64_t nloc, int64_t lda, int bw)
{
  std::vector<double> G ((size_t) bw * bw);
  int bm = (int) nloc, bn = bw, blda = (int) lda, info;
  double one = 1.0, zero = 0.0;
  for (int pass = 0; pass < 2; pass++) {
    scipy_dgemm_ ("T", "N", &bn, &bn, &bm, &one, pa, &blda, pa, &blda, &zero,
                  G.data (), &bn);
    info = 0;
    std::vector<double> G0 (G);
    scipy_dpotrf_ ("U", &bn, G.data (), &bn, &info);
    if (info != 0) {
      double dmax = 0.;
      G = G0;
      for (int i = 0; i < bw; i++) dmax = std::max (dmax, G[i + (size_t) i * bw]);
      for (int i = 0; i < bw; i++) G[i + (size_t) i * bw] += 1.e-12 * std::max (dmax, 1.);
      info = 0;
      scipy_dpotrf_ ("U", &bn, G.data (), &bn, &info);
      if (info != 0) return 76;
    }
    for (int j = 0; j < bw; j++)
      for (int i = j + 1; i < bw; i++) G[i + (size_t) j * bw] = 0.;
    scipy_dtrsm_ ("R", "U", "N", "N", &bm, &bn, &one, G.data (), &bn, pa, &blda);
  }
  return 0;
}

/* BCGS2: orthonormalize columns [p_start, ell) of Y against [0, p_start)
 * and each other, in panels of b (glr_scalapack_impl.h:153-195) */
static int
bcgs2 (double *ya, int64_t nloc, int ell, int b, int p_start)
{
  std::vector<double> C ((size_t) ell * b);
  for (int p0 = p_start; p0 < ell; p0 += b) {
    const int bw = std::min (b, ell - p0);
    double *pa = ya + (size_t) p0 * nloc;
    for (int sweep = 0; sweep < 2; sweep++) {
      if (p0 > 0) {
        int bm = (int) nloc, bj = p0, bb = bw, blda = (int) nloc;
        double one = 1.0, zero = 0.0, mone = -1.0;
        scipy_dgemm_ ("T", "N", &bj, &bb, &bm, &one, ya, &blda, pa, &blda,
                      &zero, C.data (), &bj);
        scipy_dgemm_ ("N", "N", &bm, &bb, &bj, &mone, ya, &blda, C.data (),
                      &bj, &one, pa, &blda);
      }
      int rc = panel_cholqr (pa, nloc, nloc, bw);
      if (rc) return rc;
    }
  }
  return 0;
}

/* eigensolve + |lam| ordering + truncation + treatment + U = Q C_kept
 * (glr_common_impl.h:490-574; selection as glr_scalapack_impl.h:375-425).
 * A is the raw ell x ell projection; it is symmetrized here. */
static int
rayleigh_ritz_select (orc_glr *g, int ell, const double *Q,
                      const double *Araw, orc_glr_report_t *rep,
                      std::vector<double> *evals_out,
                      std::vector<int> *order_out)
{
  const int64_t n = g->n;
  std::vector<double> T (Araw, Araw + (size_t) ell * ell), evals (ell);
  for (int j = 0; j < ell; j++)
    for (int i = 0; i < j; i++) {
      double avg = 0.5 * (T[i + (size_t) j * ell] + T[j + (size_t) i * ell]);
      T[i + (size_t) j * ell] = avg; T[j + (size_t) i * ell] = avg;
    }
  double t0 = now_s ();
  if (orc_dsyevd (ell, T.data (), evals.data (), 1) != 0) return 76;
  rep->t_dense += now_s () - t0;

  std::vector<int> order (ell);
  for (int i = 0; i < ell; i++) order[i] = i;
  for (int i = 0; i < ell; i++)
    for (int j = i + 1; j < ell; j++)
      if (fabs (evals[order[j]]) > fabs (evals[order[i]])) {
        int t = order[i]; order[i] = order[j]; order[j] = t;
      }
  double absmax = fabs (evals[order[0]]);
  double cut = 0.;
  if (g->opts.trunc_abs > 0.) cut = std::max (cut, g->opts.trunc_abs);
  if (g->opts.trunc_rel > 0.) cut = std::max (cut, g->opts.trunc_rel * absmax);
  int kept = 0;
  while (kept < ell && fabs (evals[order[kept]]) > cut) kept++;
  rep->kept = kept;
  rep->lam_abs_max = absmax;
  rep->next_abs = (kept < ell) ? fabs (evals[order[kept]]) : 0.;
  if (g->cap > 0 && kept > g->cap) {
    /* rank cap: the cap largest |lambda|; the first mode it cuts, treated,
     * becomes next_abs */
    kept = g->cap;
    rep->kept = kept;
    const double l = evals[order[kept]];
    rep->next_abs = fabs (g->opts.treat == 1 ? std::max (l, 0.) : l);
  }
  rep->lam_raw_max = evals[ell - 1];
  rep->lam_raw_min = evals[0];
  rep->n_negative_raw = 0;
  for (int i = 0; i < ell; i++)
    if (evals[i] < 0.) rep->n_negative_raw++;

  g->lam.assign (std::max (kept, 1), 0.);
  std::vector<double> C ((size_t) ell * std::max (kept, 1));
  for (int j = 0; j < kept; j++) {
    double l = evals[order[j]];
    for (int i = 0; i < ell; i++) C[i + (size_t) j * ell] = T[i + (size_t) order[j] * ell];
    switch (g->opts.treat) {
    case 0: g->lam[j] = fabs (l); break;
    case 1: g->lam[j] = std::max (l, 0.); break;
    default: g->lam[j] = l; break;
    }
  }
  g->U.assign ((size_t) n * std::max (kept, 1), 0.);
  if (kept > 0) {
    int bm = (int) n, bk = kept, bn = ell;
    double one = 1.0, zero = 0.0;
    scipy_dgemm_ ("N", "N", &bm, &bk, &bn, &one, Q, &bm, C.data (), &bn,
                  &zero, g->U.data (), &bm);
  }
  g->kept = kept;
  if (evals_out) *evals_out = evals;
  if (order_out) *order_out = order;
  return 0;
}

/* replicated build (glr_common_impl.h:414-608) as a resumable sequence of
 * pieces.  The reference's build is one call; it is restated here as a
 * state machine so that a caller can advance it one bounded piece at a
 * time (one sketch, one wave of F-apply columns, one CholQR2, the
 * Rayleigh-Ritz step, one wave of the residual check).  Every Z-solve and
 * B product is per column, so splitting an F-apply into column waves gives
 * the same bits as the whole block; orc_glr_compute runs the same machine
 * with one wave per F-apply. */
enum { BLD_SKETCH, BLD_F, BLD_ORTH, BLD_RR, BLD_CHECK, BLD_DONE };

struct orc_build
{
  orc_glr *g;
  orc_glr_report_t rep;
  int wave;  /* F-apply columns per piece */
  int phase;
  int fpass; /* which F-apply of the build: 0 .. q_power + 1 */
  int col;   /* next column of the current F-apply */
  int rc;
  std::vector<double> Q, Y, FU, evals;
  std::vector<int> order;
};

static void
build_init (orc_build *b, orc_glr *g, int wave)
{
  b->g = g;
  memset (&b->rep, 0, sizeof (b->rep));
  b->wave = wave > 0 ? wave : g->opts.ell;
  b->phase = BLD_SKETCH;
  b->fpass = 0;
  b->col = 0;
  b->rc = 0;
}

/* one piece; returns 1 while pieces remain, 0 when done, or an error code
 * (negated) */
static int
build_step (orc_build *b)
{
  orc_glr *g = b->g;
  const int ell = g->opts.ell;
  const int64_t n = g->n;
  orc_glr_report_t *rep = &b->rep;
  double t0 = now_s ();
  switch (b->phase) {
  case BLD_SKETCH:
    b->Q.assign ((size_t) n * ell, 0.);
    b->Y.assign ((size_t) n * ell, 0.);
    orc_sketch (g->opts.seed, n, 0, ell, b->Q.data ());
    b->phase = BLD_F;
    b->fpass = 0;
    b->col = 0;
    return 1;
  case BLD_F: {
    const int m = std::min (b->wave, ell - b->col);
    apply_F_block (g, m, b->Q.data () + (size_t) b->col * n,
                   b->Y.data () + (size_t) b->col * n);
    rep->t_operator += now_s () - t0;
    b->col += m;
    if (b->col < ell) return 1;
    b->col = 0;
    /* F(Omega), then q_power power passes, then the projection pass */
    b->phase = (b->fpass < g->opts.q_power + 1) ? BLD_ORTH : BLD_RR;
    return 1;
  }
  case BLD_ORTH:
    if (cholqr2 (n, ell, b->Y.data ())) { b->rc = 76; return -76; }
    rep->t_dense += now_s () - t0;
    b->Q.swap (b->Y); /* Q = Y; Y is rewritten whole by the next F-apply */
    b->fpass++;
    b->phase = BLD_F;
    return 1;
  case BLD_RR: {
    std::vector<double> A ((size_t) ell * ell);
    int bm = (int) n, bn = ell;
    double one = 1.0, zero = 0.0;
    scipy_dgemm_ ("T", "N", &bn, &bn, &bm, &one, b->Q.data (), &bm,
                  b->Y.data (), &bm, &zero, A.data (), &bn);
    int rc = rayleigh_ritz_select (g, ell, b->Q.data (), A.data (), rep,
                                   &b->evals, &b->order);
    if (rc) { b->rc = rc; return -rc; }
    if (g->incremental) { g->Q.swap (b->Q); g->A.swap (A); }
    std::vector<double> ().swap (b->Y);
    if (g->opts.check && g->kept > 0) {
      b->FU.assign ((size_t) n * g->kept, 0.);
      b->col = 0;
      b->phase = BLD_CHECK;
      return 1;
    }
    b->phase = BLD_DONE;
    return 0;
  }
  case BLD_CHECK: {
    const int kept = g->kept;
    const int m = std::min (b->wave, kept - b->col);
    apply_F_block (g, m, g->U.data () + (size_t) b->col * n,
                   b->FU.data () + (size_t) b->col * n);
    rep->t_operator += now_s () - t0;
    b->col += m;
    if (b->col < kept) return 1;
    /* residual check: max_j ||F u_j - lam_raw_j u_j|| (:576-600) */
    for (int j = 0; j < kept; j++) {
      double lraw = b->evals[b->order[j]], s = 0.;
      for (int64_t i = 0; i < n; i++) {
        double d = b->FU[i + (size_t) j * n] - lraw * g->U[i + (size_t) j * n];
        s += d * d;
      }
      rep->resid_max = std::max (rep->resid_max, sqrt (s));
    }
    std::vector<double> ().swap (b->FU);
    b->phase = BLD_DONE;
    return 0;
  }
  default:
    return 0;
  }
}

static int
build_replicated (orc_glr *g, orc_glr_report_t *rep)
{
  orc_build b;
  build_init (&b, g, 0);
  int st;
  while ((st = build_step (&b)) == 1) {}
  if (st < 0) return -st;
  *rep = b.rep;
  return 0;
}

/* incremental extension (glr_scalapack_impl.h:689-915), U materialized */
static int
extend_incremental (orc_glr *g, int k_new, orc_glr_report_t *rep)
{
  const int64_t n = g->n;
  const int ell1 = g->opts.ell, ell2 = ell1 + k_new;
  const int panel_b = g->opts.panel;
  memset (rep, 0, sizeof (*rep));
  std::vector<double> Qb ((size_t) n * ell2), Qn ((size_t) n * k_new),
      Yn ((size_t) n * k_new);
  memcpy (Qb.data (), g->Q.data (), sizeof (double) * n * ell1);
  orc_sketch (g->opts.seed, n, ell1, k_new, Qn.data ());
  double t0 = now_s ();
  apply_F_block (g, k_new, Qn.data (), Yn.data ());
  rep->t_operator += now_s () - t0;
  for (int p = 0; p < g->opts.q_power; p++) {
    t0 = now_s ();
    if (bcgs2 (Yn.data (), n, k_new, panel_b, 0)) return 76;
    rep->t_dense += now_s () - t0;
    Qn = Yn;
    t0 = now_s ();
    apply_F_block (g, k_new, Qn.data (), Yn.data ());
    rep->t_operator += now_s () - t0;
  }
  memcpy (Qb.data () + (size_t) n * ell1, Yn.data (), sizeof (double) * n * k_new);
  t0 = now_s ();
  if (bcgs2 (Qb.data (), n, ell2, panel_b, ell1)) return 76;
  rep->t_dense += now_s () - t0;
  memcpy (Qn.data (), Qb.data () + (size_t) n * ell1, sizeof (double) * n * k_new);
  t0 = now_s ();
  apply_F_block (g, k_new, Qn.data (), Yn.data ());
  rep->t_operator += now_s () - t0;
  std::vector<double> Cnew ((size_t) ell2 * k_new);
  {
    int bm = (int) n, bl2 = ell2, bk = k_new;
    double one = 1.0, zero = 0.0;
    scipy_dgemm_ ("T", "N", &bl2, &bk, &bm, &one, Qb.data (), &bm, Yn.data (),
                  &bm, &zero, Cnew.data (), &bl2);
  }
  /* grow A by symmetry (glr_scalapack_impl.h:819-840) */
  std::vector<double> A2 ((size_t) ell2 * ell2);
  for (int j = 0; j < ell1; j++) {
    for (int i = 0; i < ell1; i++)
      A2[i + (size_t) j * ell2] = g->A[i + (size_t) j * ell1];
    for (int i = ell1; i < ell2; i++)
      A2[i + (size_t) j * ell2] = Cnew[j + (size_t) (i - ell1) * ell2];
  }
  for (int j = ell1; j < ell2; j++)
    for (int i = 0; i < ell2; i++)
      A2[i + (size_t) j * ell2] = Cnew[i + (size_t) (j - ell1) * ell2];
  g->opts.ell = ell2;
  std::vector<double> evals;
  std::vector<int> order;
  int rc = rayleigh_ritz_select (g, ell2, Qb.data (), A2.data (), rep, &evals,
                                 &order);
  if (rc) return rc;
  g->Q.swap (Qb);
  g->A.swap (A2);
  return 0;
}

static orc_glr *
glr_new (const orc_csr *B, orc_prior *prior, const orc_glr_opts_t *opts,
         int incremental, int cap)
{
  orc_glr *g = new orc_glr;
  g->n = B->n;
  g->B = B;
  g->prior = prior;
  prior_ref (prior);
  g->opts = *opts;
  g->incremental = incremental;
  g->kept = 0;
  g->cap = cap > 0 ? cap : 0;
  return g;
}

extern "C" int
orc_glr_compute_cap (const orc_csr *B, orc_prior *prior,
                     const orc_glr_opts_t *opts, int incremental, int cap,
                     orc_glr **out, orc_glr_report_t *report)
{
  orc_glr_report_t rep;
  /* 0 < ell <= N (glr_common_impl.h:651-654) */
  if (opts->ell <= 0 || opts->ell > B->n) return 63;
  orc_glr *g = glr_new (B, prior, opts, incremental, cap);
  int rc = build_replicated (g, &rep);
  if (rc) { orc_prior_destroy (prior); delete g; return rc; }
  if (report) *report = rep;
  *out = g;
  return 0;
}

extern "C" int
orc_glr_compute (const orc_csr *B, orc_prior *prior,
                 const orc_glr_opts_t *opts, int incremental, orc_glr **out,
                 orc_glr_report_t *report)
{
  return orc_glr_compute_cap (B, prior, opts, incremental, 0, out, report);
}

/* The same build, advanced by the caller one piece at a time: begin, then
 * step until it returns 0 (negative: the error code of the failed step,
 * negated), then finish, which hands over the object and the report.
 * `wave` = F-apply columns per piece (0: a whole F-apply per piece). */
extern "C" orc_build *
orc_build_begin (const orc_csr *B, orc_prior *prior,
                 const orc_glr_opts_t *opts, int incremental, int cap,
                 int wave)
{
  if (opts->ell <= 0 || opts->ell > B->n) return NULL;
  orc_build *b = new orc_build;
  build_init (b, glr_new (B, prior, opts, incremental, cap), wave);
  return b;
}

extern "C" int
orc_build_step (orc_build *b)
{
  return build_step (b);
}

extern "C" orc_glr *
orc_build_finish (orc_build *b, orc_glr_report_t *report)
{
  orc_glr *g = b->g;
  if (b->phase != BLD_DONE || b->rc) {
    orc_prior_destroy (g->prior);
    delete g;
    g = NULL;
  } else if (report) {
    *report = b->rep;
  }
  delete b;
  return g;
}

/* glr_common_impl.h:684-719 */
extern "C" int
orc_glr_extend (orc_glr *g, int k_new, orc_glr_report_t *report)
{
  orc_glr_report_t rep;
  if (k_new <= 0) return 63;
  if (g->opts.ell + k_new > g->n) return 63;
  int rc;
  if (g->incremental) rc = extend_incremental (g, k_new, &rep);
  else {
    g->opts.ell += k_new;
    rc = build_replicated (g, &rep);
  }
  if (rc) return rc;
  if (report) *report = rep;
  return 0;
}

extern "C" void
orc_glr_destroy (orc_glr *g)
{
  if (!g) return;
  orc_prior_destroy (g->prior);
  delete g;
}

extern "C" int
orc_glr_eigs (const orc_glr *g, int *nkept, const double **lam)
{
  *nkept = g->kept;
  *lam = g->lam.data ();
  return 0;
}

extern "C" const double *
orc_glr_U (const orc_glr *g)
{
  return g->U.data ();
}

/* ---- downstream (glr_common_impl.h:747-1104) ------------------------- */

/* out = f_c in + U diag(f_lam - f_c) U^T in (glr_common_impl.h:948-966) */
static void
filter_core (const orc_glr *g, const double *f_lam, double f_c,
             const double *in, double *out)
{
  const int64_t n = g->n;
  if (g->kept == 0) {
    for (int64_t i = 0; i < n; i++) out[i] = f_c * in[i];
    return;
  }
  std::vector<double> w (g->kept);
  int bm = (int) n, bk = g->kept, ione = 1;
  double one = 1.0, zero = 0.0;
  scipy_dgemv_ ("T", &bm, &bk, &one, g->U.data (), &bm, in, &ione, &zero,
                w.data (), &ione);
  for (int k = 0; k < g->kept; k++) w[k] *= f_lam[k] - f_c;
  for (int64_t i = 0; i < n; i++) out[i] = f_c * in[i];
  scipy_dgemv_ ("N", &bm, &bk, &one, g->U.data (), &bm, w.data (), &ione,
                &one, out, &ione);
}

/* block master formula (glr_common_impl.h:910-929), column-major n x m */
extern "C" void
orc_glr_filter_block (const orc_glr *g, const double *f_lam, double f_c,
                      int m, const double *X, double *Y)
{
  const int64_t n = g->n;
  for (size_t i = 0; i < (size_t) n * m; i++) Y[i] = f_c * X[i];
  if (g->kept == 0) return;
  std::vector<double> W ((size_t) g->kept * m);
  int bm = (int) n, bk = g->kept, bmm = m;
  double one = 1.0, zero = 0.0;
  scipy_dgemm_ ("T", "N", &bk, &bmm, &bm, &one, g->U.data (), &bm, X, &bm,
                &zero, W.data (), &bk);
  for (int j = 0; j < m; j++)
    for (int k = 0; k < g->kept; k++) W[k + (size_t) j * g->kept] *= f_lam[k] - f_c;
  scipy_dgemm_ ("N", "N", &bm, &bmm, &bk, &one, g->U.data (), &bm, W.data (),
                &bk, &one, Y, &bm);
}

extern "C" int
orc_glr_filter (const orc_glr *g, const double *f_lam, double f_c,
                const double *in, double *out)
{
  filter_core (g, f_lam, f_c, in, out);
  return 0;
}

extern "C" int
orc_glr_pow (const orc_glr *g, double c, double p, const double *in,
             double *out)
{
  if (!(c > 0.)) return 63;
  std::vector<double> f (std::max (g->kept, 1));
  for (int i = 0; i < g->kept; i++) f[i] = pow (g->lam[i] + c, p);
  filter_core (g, f.data (), pow (c, p), in, out);
  return 0;
}

/* glr_common_impl.h:988-997 */
extern "C" double
orc_glr_logdet (const orc_glr *g, double c)
{
  double s = 0.;
  for (int i = 0; i < g->kept; i++) s += log (g->lam[i] + c) - log (c);
  return s;
}

/* glr_common_impl.h:1007-1024 */
extern "C" int
orc_glr_solve (orc_glr *g, double c, const double *rhs, double *x)
{
  const int64_t n = g->n;
  if (!(c > 0.)) return 63;
  std::vector<double> w1 (n), w2 (n), f (std::max (g->kept, 1));
  orc_prior_solveZ (g->prior, rhs, w1.data ());
  for (int64_t i = 0; i < n; i++) w1[i] *= g->prior->msqrt[i];
  for (int i = 0; i < g->kept; i++) f[i] = 1. / (g->lam[i] + c);
  filter_core (g, f.data (), 1. / c, w1.data (), w2.data ());
  for (int64_t i = 0; i < n; i++) w2[i] *= g->prior->msqrt[i];
  orc_prior_solveZ (g->prior, w2.data (), x);
  return 0;
}

/* lgh_glr_solve (glr_common_impl.h:1007-1024) on m right-hand sides at
 * one shift, column-major n x m: the two Z-solves run column-parallel
 * (orc_prior_solve_block), the master formula as one block product
 * (glr_common_impl.h:910-929).  Per column the same arithmetic as m calls
 * of orc_glr_solve, with the BLAS-2 passes over U batched into BLAS-3. */
extern "C" int
orc_glr_solve_block (orc_glr *g, double c, int m, const double *rhs,
                     double *x)
{
  const int64_t n = g->n;
  if (!(c > 0.)) return 63;
  std::vector<double> W1 ((size_t) n * m), W2 ((size_t) n * m),
      f (std::max (g->kept, 1));
  orc_prior_solve_block (g->prior, m, rhs, W1.data ());
  for (int j = 0; j < m; j++)
    for (int64_t i = 0; i < n; i++) W1[i + (size_t) j * n] *= g->prior->msqrt[i];
  for (int i = 0; i < g->kept; i++) f[i] = 1. / (g->lam[i] + c);
  orc_glr_filter_block (g, f.data (), 1. / c, m, W1.data (), W2.data ());
  for (int j = 0; j < m; j++)
    for (int64_t i = 0; i < n; i++) W2[i + (size_t) j * n] *= g->prior->msqrt[i];
  orc_prior_solve_block (g->prior, m, W2.data (), x);
  return 0;
}

/* exact y = B v + c R v (glr_common_impl.h:1026-1048, uncorrected) */
extern "C" int
orc_glr_apply (orc_glr *g, double c, const double *v, double *y)
{
  const int64_t n = g->n;
  std::vector<double> w (n);
  csr_mult_par (g->B, v, y);
  orc_prior_apply (g->prior, v, w.data ());
  for (int64_t i = 0; i < n; i++) y[i] += c * w[i];
  return 0;
}

/* glr_common_impl.h:1050-1097 */
extern "C" int
orc_glr_factor (orc_glr *g, double c, int which, const double *in,
                double *out)
{
  const int64_t n = g->n;
  if (!(c > 0.)) return 63;
  std::vector<double> w1 (n), f (std::max (g->kept, 1));
  switch (which) {
  case 0: /* G = Z M^{-1/2} S */
    for (int i = 0; i < g->kept; i++) f[i] = pow (g->lam[i] + c, 0.5);
    filter_core (g, f.data (), sqrt (c), in, w1.data ());
    for (int64_t i = 0; i < n; i++) w1[i] *= g->prior->minvsqrt[i];
    orc_prior_applyZ (g->prior, w1.data (), out);
    break;
  case 1: /* GT = S M^{-1/2} Z^T */
    orc_prior_applyZ (g->prior, in, w1.data ());
    for (int64_t i = 0; i < n; i++) w1[i] *= g->prior->minvsqrt[i];
    for (int i = 0; i < g->kept; i++) f[i] = pow (g->lam[i] + c, 0.5);
    filter_core (g, f.data (), sqrt (c), w1.data (), out);
    break;
  case 2: /* GINV = S^{-1} M^{1/2} Z^{-1} */
    orc_prior_solveZ (g->prior, in, w1.data ());
    for (int64_t i = 0; i < n; i++) w1[i] *= g->prior->msqrt[i];
    for (int i = 0; i < g->kept; i++) f[i] = 1. / pow (g->lam[i] + c, 0.5);
    filter_core (g, f.data (), 1. / sqrt (c), w1.data (), out);
    break;
  case 3: /* GINVT = Z^{-T} M^{1/2} S^{-1} */
    for (int i = 0; i < g->kept; i++) f[i] = 1. / pow (g->lam[i] + c, 0.5);
    filter_core (g, f.data (), 1. / sqrt (c), in, w1.data ());
    for (int64_t i = 0; i < n; i++) w1[i] *= g->prior->msqrt[i];
    orc_prior_solveZ (g->prior, w1.data (), out);
    break;
  default:
    return 63;
  }
  return 0;
}

/* glr_common_impl.h:1099-1104 */
extern "C" int
orc_glr_sample (orc_glr *g, double c, const double *xi, double *x)
{
  return orc_glr_factor (g, c, 3, xi, x);
}

/* one F-apply of m columns on the object's operator: used by the
 * CPU-baseline timing leg to time the per-column operator cost. */
extern "C" void
orc_glr_apply_F (orc_glr *g, int m, const double *X, double *Y)
{
  apply_F_block (g, m, X, Y);
}

/* a bare build context for timing F-applies without a full build */
extern "C" orc_glr *
orc_glr_context (const orc_csr *B, orc_prior *prior)
{
  orc_glr *g = new orc_glr;
  g->n = B->n;
  g->B = B;
  g->prior = prior;
  prior_ref (prior);
  memset (&g->opts, 0, sizeof (g->opts));
  g->incremental = 0;
  g->kept = 0;
  return g;
}

/* dense building blocks exposed for the CPU-baseline leg (timed at the
 * full ell on the host): CholQR2 and the Rayleigh-Ritz eigensolve. */
extern "C" int
orc_cholqr2 (int64_t n, int ncols, double *X)
{
  return cholqr2 (n, ncols, X);
}
