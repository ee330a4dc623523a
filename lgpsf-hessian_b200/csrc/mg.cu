/* mg.cu -- aggregation multigrid for the Z-solves: the device counterpart
 * of the reference's PCGAMG preconditioner (zsolve_impl.h:808-818) and of
 * its mode-3 block V-cycle on the harvested hierarchy (zsolve_impl.h:
 * 198-485).
 *
 * Setup (host, once per prior; PCSetUp's role): smoothed aggregation from
 * Z's CSR -- greedy aggregates of the strength graph, the constant
 * near-null space, tentative prolongator smoothed by one damped Jacobi step
 * (omega = 4/3 / lambda_max(D^{-1} A)), Galerkin coarse operators
 * A_c = P^T A P, until the coarse size drops below a few thousand; the
 * coarsest operator is inverted densely on the device (Cholesky + inverse
 * factor, the reference's dense-LU coarse solve).  Per level, the smoothing
 * interval [0.1, smoother_top] * lambda_max(D^{-1} A_l) from CG-Lanczos
 * (zsolve_impl.h:284-313, 340-341) and nu = 2 Chebyshev-Jacobi terms.
 *
 * Solve (device): the block V-cycle in correction form, every operation on
 * row-major blocks: Chebyshev-Jacobi pre-smoothing (the fused k_cheb kernel
 * keeps the residual current), restriction R_c = P^T R (CSR of P^T),
 * recursion, prolongation X += P X_c and the residual refresh R = B - A X
 * (the accumulate and residual forms of the row-group CSR product),
 * post-smoothing; coarse level X = A_0^{-1} B as a dense product.
 */

#include <math.h>
#include <string.h>

#include <omp.h>

#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "lgh_device.cuh"
#include "lgh_internal.h"
#include "lgh_ktime.h"
#include "lgh_mg.h"

namespace lgh
{

/* ---- host CSR helpers -------------------------------------------------- */

/* an allocator whose resize leaves new elements uninitialised: every
 * column and value array of the host set-up is sized and then written in
 * full by a parallel loop (or a copy), so its pages are first touched by
 * the threads that fill them instead of by a serial zero fill */
template <typename T>
struct NoInitAlloc : std::allocator<T>
{
  template <typename U> struct rebind { using other = NoInitAlloc<U>; };
  NoInitAlloc () = default;
  template <typename U> NoInitAlloc (const NoInitAlloc<U> &) noexcept {}
  template <typename U> void construct (U *p) noexcept { ::new ((void *) p) U; }
  template <typename U, typename... Args>
  void construct (U *p, Args &&...args)
  {
    ::new ((void *) p) U (std::forward<Args> (args)...);
  }
};

struct HCsr
{
  int64_t n = 0, m = 0; /* rows, cols */
  std::vector<int64_t> rp;
  std::vector<int32_t, NoInitAlloc<int32_t>> ci;
  std::vector<double, NoInitAlloc<double>> v;
};

static double
hcsr_diag (const HCsr &A, int64_t i)
{
  for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++)
    if (A.ci[k] == i) return A.v[k];
  return 0.;
}

/* The host set-up runs its row loops on all host threads (OpenMP); every
 * reduction sums fixed row blocks in a fixed order, so the hierarchy is
 * the same bits whatever the thread count. */
static void
hcsr_mult (const HCsr &A, const std::vector<double> &x, std::vector<double> &y)
{
  y.assign (A.n, 0.);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A.n; i++) {
    double s = 0.;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++) s += A.v[k] * x[A.ci[k]];
    y[i] = s;
  }
}

/* sum_i a_i b_i over 256 fixed row blocks, combined in order */
static double
hdot (const std::vector<double> &a, const std::vector<double> &b)
{
  const int64_t n = (int64_t) a.size ();
  constexpr int NB = 256;
  double part[NB];
#pragma omp parallel for schedule(static)
  for (int blk = 0; blk < NB; blk++) {
    const int64_t i0 = n * blk / NB, i1 = n * (blk + 1) / NB;
    double s = 0.;
    for (int64_t i = i0; i < i1; i++) s += a[i] * b[i];
    part[blk] = s;
  }
  double s = 0.;
  for (int blk = 0; blk < NB; blk++) s += part[blk];
  return s;
}

/* T = A^T with each row of T in ascending source row order.  Row chunks
 * of A count their entries per column, the counts give every chunk its
 * start in each row of T (chunks in row order), and the chunks scatter
 * in parallel: the result is the serial transpose's, bit for bit. */
static HCsr
hcsr_transpose (const HCsr &A)
{
  HCsr T;
  T.n = A.m;
  T.m = A.n;
  const int64_t nnz = A.rp[A.n];
  T.rp.assign (T.n + 1, 0);
  T.ci.resize (nnz);
  T.v.resize (nnz);
  const int nt = std::max (1, std::min (omp_get_max_threads (), 64));
  /* one chunk per thread, unless the count arrays would outweigh A */
  int nch = (int) std::min<int64_t> (std::max<int64_t> (A.n, 1), nt);
  while (nch > 1 && (int64_t) nch * T.n > 4 * nnz + 4096) nch /= 2;
  std::vector<int64_t> pos ((size_t) nch * T.n, 0);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int c = 0; c < nch; c++) {
    int64_t *cnt = pos.data () + (size_t) c * T.n;
    const int64_t r0 = A.n * c / nch, r1 = A.n * (c + 1) / nch;
    for (int64_t k = A.rp[r0]; k < A.rp[r1]; k++) cnt[A.ci[k]]++;
  }
  /* row starts of T, then each chunk's start within every row */
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t j = 0; j < T.n; j++) {
    int64_t s = 0;
    for (int c = 0; c < nch; c++) s += pos[(size_t) c * T.n + j];
    T.rp[j + 1] = s;
  }
  for (int64_t j = 0; j < T.n; j++) T.rp[j + 1] += T.rp[j];
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t j = 0; j < T.n; j++) {
    int64_t s = T.rp[j];
    for (int c = 0; c < nch; c++) {
      const int64_t k = pos[(size_t) c * T.n + j];
      pos[(size_t) c * T.n + j] = s;
      s += k;
    }
  }
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int c = 0; c < nch; c++) {
    int64_t *at = pos.data () + (size_t) c * T.n;
    const int64_t r0 = A.n * c / nch, r1 = A.n * (c + 1) / nch;
    for (int64_t i = r0; i < r1; i++)
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++) {
        const int64_t p = at[A.ci[k]]++;
        T.ci[p] = (int32_t) i;
        T.v[p] = A.v[k];
      }
  }
  return T;
}

/* rows of a product assembled chunk by chunk: each chunk's rows go into
 * vectors of its own (moved out once, so threads never write shared
 * headers), then the chunks are concatenated in parallel at their
 * offsets; the result does not depend on the thread count */
struct HChunk
{
  std::vector<int32_t> ci;
  std::vector<double> v;
  std::vector<int64_t> cnt;
};

static void
hcsr_concat (std::vector<HChunk> &ch, int64_t n, HCsr &C)
{
  const int nch = (int) ch.size ();
  std::vector<int64_t> off (nch + 1, 0), roff (nch + 1, 0);
  for (int c = 0; c < nch; c++) {
    off[c + 1] = off[c] + (int64_t) ch[c].ci.size ();
    roff[c + 1] = roff[c] + (int64_t) ch[c].cnt.size ();
  }
  C.rp.assign (n + 1, 0);
  C.ci.resize (off[nch]);
  C.v.resize (off[nch]);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nch; c++) {
    if (!ch[c].ci.empty ()) {
      memcpy (C.ci.data () + off[c], ch[c].ci.data (), ch[c].ci.size () * sizeof (int32_t));
      memcpy (C.v.data () + off[c], ch[c].v.data (), ch[c].v.size () * sizeof (double));
    }
    int64_t pos = off[c];
    for (size_t r = 0; r < ch[c].cnt.size (); r++) {
      pos += ch[c].cnt[r];
      C.rp[roff[c] + (int64_t) r + 1] = pos;
    }
  }
}

static HCsr
hcsr_gemm (const HCsr &A, const HCsr &B)
{
  /* C = A B (Gustavson, dense accumulator), columns sorted per row: a
   * counting pass sizes every row, then the rows are formed in place, in
   * parallel; each row sums its terms in A's then B's entry order, so the
   * product does not depend on the thread count */
  HCsr C;
  C.n = A.n;
  C.m = B.m;
  const int nt = std::max (1, std::min (omp_get_max_threads (), 64));
  /* about 8 scheduling chunks per thread, at least 64 rows each */
  const int64_t rows_per = std::max<int64_t> (64, A.n / (8 * nt));
  C.rp.assign (C.n + 1, 0);
#pragma omp parallel num_threads(nt)
  {
    std::vector<int64_t> mark (B.m, -1);
#pragma omp for schedule(dynamic, rows_per)
    for (int64_t i = 0; i < A.n; i++) {
      int64_t cnt = 0;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++) {
        const int64_t j = A.ci[k];
        for (int64_t q = B.rp[j]; q < B.rp[j + 1]; q++) {
          const int32_t col = B.ci[q];
          if (mark[col] != i) {
            mark[col] = i;
            cnt++;
          }
        }
      }
      C.rp[i + 1] = cnt;
    }
  }
  for (int64_t i = 0; i < C.n; i++) C.rp[i + 1] += C.rp[i];
  C.ci.resize (C.rp[C.n]);
  C.v.resize (C.rp[C.n]);
#pragma omp parallel num_threads(nt)
  {
    std::vector<double> acc (B.m, 0.);
    std::vector<int64_t> mark (B.m, -1);
#pragma omp for schedule(dynamic, rows_per)
    for (int64_t i = 0; i < A.n; i++) {
      int32_t *cols = C.ci.data () + C.rp[i];
      size_t nc = 0;
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++) {
        const int64_t j = A.ci[k];
        const double a = A.v[k];
        for (int64_t q = B.rp[j]; q < B.rp[j + 1]; q++) {
          const int32_t col = B.ci[q];
          if (mark[col] != i) {
            mark[col] = i;
            acc[col] = 0.;
            cols[nc++] = col;
          }
          acc[col] += a * B.v[q];
        }
      }
      /* ascending columns: rows of these products hold a few dozen
       * entries at most, where an insertion sort beats std::sort */
      if (nc > 48) {
        std::sort (cols, cols + nc);
      } else {
        for (size_t t = 1; t < nc; t++) {
          const int32_t x = cols[t];
          size_t u = t;
          for (; u > 0 && cols[u - 1] > x; u--) cols[u] = cols[u - 1];
          cols[u] = x;
        }
      }
      double *v = C.v.data () + C.rp[i];
      for (size_t t = 0; t < nc; t++) v[t] = acc[cols[t]];
    }
  }
  return C;
}

static double lanczos_tail (const std::vector<double> &al,
                            const std::vector<double> &be);

/* lambda_max(D^{-1} A) from CG-Lanczos with Jacobi (its steps, fixed
 * hashed probe), the estimate of zsolve_impl.h:284-313; extremal
 * eigenvalue of the tridiagonal by Sturm bisection */
static double
lanczos_lmax (const HCsr &A, int its, uint64_t seed)
{
  const int64_t n = A.n;
  std::vector<double> dinv (n), r (n), z (n), p (n), q (n), x (n, 0.);
  for (int64_t i = 0; i < n; i++) {
    const double d = hcsr_diag (A, i);
    dinv[i] = d != 0. ? 1. / d : 0.;
    r[i] = 0.5 - (double) ((rng_state_at (seed, i, 0) >> 11) * (1.0 / 9007199254740992.0));
  }
  std::vector<double> al, be;
  double rz = 0., rzold = 0.;
  for (int64_t i = 0; i < n; i++) z[i] = dinv[i] * r[i];
  rz = hdot (r, z);
  p = z;
  for (int k = 0; k < its; k++) {
    hcsr_mult (A, p, q);
    const double pq = hdot (p, q);
    if (!(pq > 0.)) break;
    const double a = rz / pq;
    al.push_back (a);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      x[i] += a * p[i];
      r[i] -= a * q[i];
      z[i] = dinv[i] * r[i];
    }
    rzold = rz;
    rz = hdot (r, z);
    if (rz <= 1e-300) break;
    const double b = rz / rzold;
    be.push_back (b);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) p[i] = z[i] + b * p[i];
  }
  return lanczos_tail (al, be);
}

/* the largest eigenvalue of the Lanczos tridiagonal of a CG run with step
 * lengths al (alpha) and be (beta): bisection on the Sturm count */
static double
lanczos_tail (const std::vector<double> &al, const std::vector<double> &be)
{
  const int m = (int) al.size ();
  if (m == 0) return 2.0;
  std::vector<double> d (m), e (m, 0.);
  for (int k = 0; k < m; k++) {
    d[k] = 1. / al[k] + (k > 0 ? be[k - 1] / al[k - 1] : 0.);
    if (k + 1 < m) e[k] = sqrt (fabs (be[k])) / al[k];
  }
  /* Gershgorin upper bound, then bisection on the Sturm count */
  double hi = 0.;
  for (int k = 0; k < m; k++)
    hi = std::max (hi, d[k] + fabs (e[k]) + (k > 0 ? fabs (e[k - 1]) : 0.));
  double lo = 0.;
  for (int it = 0; it < 200; it++) {
    const double mid = 0.5 * (lo + hi);
    int cnt = 0;  /* eigenvalues > mid */
    double t = d[0] - mid;
    if (t > 0.) cnt++;
    for (int k = 1; k < m; k++) {
      const double den = (t != 0.) ? t : 1e-300;
      t = d[k] - mid - e[k - 1] * e[k - 1] / den;
      if (t > 0.) cnt++;
    }
    if (cnt >= 1) lo = mid;
    else hi = mid;
  }
  return hi;
}

/* one smoothed-aggregation coarsening step */
static void
sa_coarsen (const HCsr &A, double theta, double lmax, HCsr &P, int64_t &nc)
{
  const int64_t n = A.n;
  std::vector<double> diag (n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) diag[i] = hcsr_diag (A, i);
  auto strong = [&] (int64_t i, int64_t k) {
    const int64_t j = A.ci[k];
    return j != i && fabs (A.v[k]) > theta * sqrt (fabs (diag[i] * diag[j]));
  };
  std::vector<int64_t> agg (n, -1);
  nc = 0;
  /* pass 1: roots whose strong neighbourhood is free */
  for (int64_t i = 0; i < n; i++) {
    if (agg[i] >= 0) continue;
    bool free_nb = true;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1] && free_nb; k++)
      if (strong (i, k) && agg[A.ci[k]] >= 0) free_nb = false;
    if (!free_nb) continue;
    agg[i] = nc;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++)
      if (strong (i, k)) agg[A.ci[k]] = nc;
    nc++;
  }
  /* pass 2: attach to the strongest aggregated neighbour (pass-1 state) */
  std::vector<int64_t> agg1 = agg;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    if (agg1[i] >= 0) continue;
    double best = -1.;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++)
      if (strong (i, k) && agg1[A.ci[k]] >= 0 && fabs (A.v[k]) > best) {
        best = fabs (A.v[k]);
        agg[i] = agg1[A.ci[k]];
      }
  }
  /* pass 3: leftovers become singletons */
  for (int64_t i = 0; i < n; i++)
    if (agg[i] < 0) agg[i] = nc++;
  /* tentative prolongator (constant near-null space, orthonormal cols) */
  std::vector<double> sz (nc, 0.);
  for (int64_t i = 0; i < n; i++) sz[agg[i]] += 1.;
  std::vector<double> p0 (n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) p0[i] = 1. / sqrt (sz[agg[i]]);
  /* omega = 4/3 / lambda_max(D^{-1}A) (the level's own estimate) */
  const double omega = (4.0 / 3.0) / lmax;
  /* P = (I - omega D^{-1} A) P0, rows in parallel chunks */
  P.n = n;
  P.m = nc;
  const int nt = std::max (1, std::min (omp_get_max_threads (), 64));
  const int nchunk = (int) std::min<int64_t> (std::max<int64_t> (n, 1), 4 * nt);
  std::vector<HChunk> ch (nchunk);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int c = 0; c < nchunk; c++) {
    const int64_t r0 = n * c / nchunk, r1 = n * (c + 1) / nchunk;
    HChunk loc;
    loc.cnt.reserve (r1 - r0);
    std::vector<int64_t> cols;
    std::vector<double> acc;
    for (int64_t i = r0; i < r1; i++) {
      cols.clear ();
      acc.clear ();
      auto add = [&] (int64_t col, double val) {
        for (size_t t = 0; t < cols.size (); t++)
          if (cols[t] == col) { acc[t] += val; return; }
        cols.push_back (col);
        acc.push_back (val);
      };
      add (agg[i], p0[i]);
      const double sc = omega / diag[i];
      for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++) {
        const int64_t j = A.ci[k];
        add (agg[j], -sc * A.v[k] * p0[j]);
      }
      /* ascending columns (insertion sort: rows hold a few aggregates) */
      for (size_t t = 1; t < cols.size (); t++)
        for (size_t u = t; u > 0 && cols[u - 1] > cols[u]; u--) {
          std::swap (cols[u - 1], cols[u]);
          std::swap (acc[u - 1], acc[u]);
        }
      int64_t kept = 0;
      for (size_t t = 0; t < cols.size (); t++) {
        if (acc[t] == 0.) continue;
        loc.ci.push_back ((int32_t) cols[t]);
        loc.v.push_back (acc[t]);
        kept++;
      }
      loc.cnt.push_back (kept);
    }
    ch[c] = std::move (loc);
  }
  hcsr_concat (ch, n, P);
}


/* ---- device kernels ------------------------------------------------------ */

/* ---- lambda_max(D^{-1} A) on the device -----------------------------------
 * The recurrence of lanczos_lmax on a level's device operator: the same
 * hashed start vector, Jacobi-preconditioned CG steps whose lengths form
 * the Lanczos tridiagonal.  Three launches per step; each reduction sums
 * fixed per-block partials in block order in the last block to finish (the
 * same bits on every run); the step lengths come back in one copy. */
constexpr int LZ_MAX = 64;
constexpr int LZ_BLOCK = 256;

struct LzState
{
  double rz;
  double alpha[LZ_MAX], beta[LZ_MAX];
  int na, nb, stop, step_ok;
  unsigned ticket;
};

/* this block's sum of v into part[blockIdx.x]; in the last block to
 * finish, thread 0 gets the total over all blocks and returns true */
__device__ bool
lz_reduce (double v, double *part, unsigned *ticket, double *total)
{
  __shared__ double red[LZ_BLOCK / 32];
  __shared__ bool last;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync (0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads ();
  if (threadIdx.x == 0) {
    double sum = 0.;
    for (int w = 0; w < LZ_BLOCK / 32; w++) sum += red[w];
    part[blockIdx.x] = sum;
    __threadfence ();
    last = atomicAdd (ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads ();
  if (!last || threadIdx.x != 0) return false;
  __threadfence ();
  double sum = 0.;
  for (unsigned b = 0; b < gridDim.x; b++) sum += ((volatile double *) part)[b];
  *total = sum;
  *ticket = 0u;
  return true;
}

__global__ void __launch_bounds__ (LZ_BLOCK)
k_lz_init (int64_t n, uint64_t seed, const double *dinv, double *r, double *z,
           double *p, double *part, LzState *st)
{
  double acc = 0.;
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x) {
    const double ri = 0.5 - (double) ((rng_state_at (seed, i, 0) >> 11)
                                      * (1.0 / 9007199254740992.0));
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    acc += ri * zi;
  }
  double tot;
  if (lz_reduce (acc, part, &st->ticket, &tot)) st->rz = tot;
}

/* q = A p, alpha = (r, z) / (p, q) */
__global__ void __launch_bounds__ (LZ_BLOCK)
k_lz_q (int64_t n, const int64_t *rp, const int32_t *ci, const double *v,
        const double *p, double *q, double *part, LzState *st)
{
  if (st->stop) return;
  double acc = 0.;
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x) {
    double sum = 0.;
    for (int64_t k = rp[i]; k < rp[i + 1]; k++) sum += v[k] * p[ci[k]];
    q[i] = sum;
    acc += p[i] * sum;
  }
  double pq;
  if (lz_reduce (acc, part, &st->ticket, &pq)) {
    if (!(pq > 0.) || st->na >= LZ_MAX) {
      st->stop = 1;
      st->step_ok = 0;
    } else {
      st->alpha[st->na++] = st->rz / pq;
      st->step_ok = 1;
    }
  }
}

/* r -= alpha q, z = D^{-1} r, beta = (r, z)_new / (r, z)_old */
__global__ void __launch_bounds__ (LZ_BLOCK)
k_lz_r (int64_t n, const double *dinv, double *r, double *z, const double *q,
        double *part, LzState *st)
{
  if (!st->step_ok) return;
  const double a = st->alpha[st->na - 1];
  double acc = 0.;
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x) {
    const double ri = r[i] - a * q[i];
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    acc += ri * zi;
  }
  double rz;
  if (lz_reduce (acc, part, &st->ticket, &rz)) {
    const double rzold = st->rz;
    st->rz = rz;
    if (rz <= 1e-300) {
      st->stop = 1;
      st->step_ok = 0;
    } else {
      st->beta[st->nb++] = rz / rzold;
    }
  }
}

/* p = z + beta p */
__global__ void __launch_bounds__ (LZ_BLOCK)
k_lz_p (int64_t n, const double *z, double *p, const LzState *st)
{
  if (!st->step_ok) return;
  const double b = st->beta[st->nb - 1];
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    p[i] = z[i] + b * p[i];
}

static int
lanczos_lmax_dev (const Csr &A, int its, uint64_t seed, double *lmax)
{
  const int64_t n = A.n;
  cudaStream_t s = stream ();
  const int grid = (int) std::max<int64_t> (1, std::min<int64_t> (
      (int64_t) num_sms () * 4, (n + LZ_BLOCK - 1) / LZ_BLOCK));
  its = std::min (its, LZ_MAX);
  DBuf<double> r, z, p, q, part;
  DBuf<char> stb;
  LGH_TRY (r.alloc (n));
  LGH_TRY (z.alloc (n));
  LGH_TRY (p.alloc (n));
  LGH_TRY (q.alloc (n));
  LGH_TRY (part.alloc (grid));
  LGH_TRY (stb.alloc (sizeof (LzState)));
  LzState *st = (LzState *) stb.p;
  LGH_CUDA (cudaMemsetAsync (st, 0, sizeof (LzState), s));
  k_lz_init<<<grid, LZ_BLOCK, 0, s>>> (n, seed, A.dinv, r.p, z.p, p.p, part.p, st);
  LGH_LAUNCH_CHECK ();
  for (int k = 0; k < its; k++) {
    k_lz_q<<<grid, LZ_BLOCK, 0, s>>> (n, A.rowptr, A.colidx, A.vals, p.p, q.p,
                                      part.p, st);
    k_lz_r<<<grid, LZ_BLOCK, 0, s>>> (n, A.dinv, r.p, z.p, q.p, part.p, st);
    k_lz_p<<<grid, LZ_BLOCK, 0, s>>> (n, z.p, p.p, st);
  }
  LGH_LAUNCH_CHECK ();
  LzState h;
  LGH_CUDA (cudaMemcpyAsync (&h, st, sizeof (LzState), cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  std::vector<double> al (h.alpha, h.alpha + h.na), be (h.beta, h.beta + h.nb);
  *lmax = lanczos_tail (al, be);
  return 0;
}

/* levels of at least this many rows estimate on the device */
constexpr int64_t LZ_DEVICE_MIN = 20000;

/* ---- host <-> device ------------------------------------------------------ */

/* upload a host CSR into a device Csr (float copy and 1/diag filled) */
static int
csr_upload (const HCsr &H, Csr &D)
{
  D = Csr ();
  D.n = H.n;
  D.ncols = H.m > 0 ? H.m : H.n;
  D.nnz = H.rp[H.n];
  LGH_TRY (dalloc ((void **) &D.rowptr, (size_t) (H.n + 1) * sizeof (int64_t)));
  LGH_TRY (dalloc ((void **) &D.colidx, (size_t) D.nnz * sizeof (int32_t) + 16));
  LGH_TRY (dalloc ((void **) &D.vals, (size_t) D.nnz * sizeof (double) + 16));
  LGH_CUDA (cudaMemcpy (D.rowptr, H.rp.data (), (H.n + 1) * sizeof (int64_t),
                        cudaMemcpyHostToDevice));
  if (D.nnz) {
    LGH_CUDA (cudaMemcpy (D.colidx, H.ci.data (), D.nnz * sizeof (int32_t),
                          cudaMemcpyHostToDevice));
    LGH_CUDA (cudaMemcpy (D.vals, H.v.data (), D.nnz * sizeof (double),
                          cudaMemcpyHostToDevice));
  }
  return csr_finish (D);
}

static int
csr_download (const Csr &D, HCsr &H)
{
  H.n = D.n;
  H.m = D.n;
  H.rp.resize (D.n + 1);
  H.ci.resize (D.nnz);
  H.v.resize (D.nnz);
  LGH_CUDA (cudaMemcpy (H.rp.data (), D.rowptr, (D.n + 1) * sizeof (int64_t),
                        cudaMemcpyDeviceToHost));
  LGH_CUDA (cudaMemcpy (H.ci.data (), D.colidx, D.nnz * sizeof (int32_t),
                        cudaMemcpyDeviceToHost));
  LGH_CUDA (cudaMemcpy (H.v.data (), D.vals, D.nnz * sizeof (double),
                        cudaMemcpyDeviceToHost));
  return 0;
}

Hierarchy::~Hierarchy ()
{
  for (auto &l : lev) {
    if (l.own) csr_free (l.A);
    csr_free (l.P);
    csr_free (l.R);
    dfree (l.f1v);
    dfree (l.f1v32);
    csr_free (l.AP);
  }
}

/* the first smoothing step's values: fl(b1 vd) and fl((float) b1 vd32) */
__global__ void
k_first_step_vals (int64_t nnz, double b1, const double *__restrict__ vd,
                   const float *__restrict__ vd32, double *__restrict__ out,
                   float *__restrict__ out32)
{
  const float b1f = (float) b1;
  for (int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
       k += (int64_t) gridDim.x * blockDim.x) {
    out[k] = b1 * vd[k];
    out32[k] = b1f * vd32[k];
  }
}

static int
first_step_operator (MgLevel &lv)
{
  const Csr &A = lv.A;
  if (!A.vd || !A.vd32 || A.nnz == 0) return 0;
  const double theta = 0.5 * (lv.shi + lv.slo);
  const double b1 = 1.0 / theta;      /* mg_smooth's first coefficient */
  int rc = dalloc ((void **) &lv.f1v, (size_t) A.nnz * sizeof (double) + 16);
  if (!rc) rc = dalloc ((void **) &lv.f1v32, (size_t) A.nnz * sizeof (float) + 16);
  if (rc) {
    dfree (lv.f1v);
    dfree (lv.f1v32);
    lv.f1v = nullptr;
    lv.f1v32 = nullptr;
    return rc;
  }
  const int grid = (int) std::max<int64_t> (1, std::min<int64_t> (
      (A.nnz + 255) / 256, (int64_t) num_sms () * 8));
  k_first_step_vals<<<grid, 256, 0, stream ()>>> (A.nnz, b1, A.vd, A.vd32,
                                                  lv.f1v, lv.f1v32);
  LGH_LAUNCH_CHECK ();
  lv.F1 = A;                          /* A's pattern; only the values differ */
  lv.F1.vals = lv.f1v;
  lv.F1.vals32 = lv.f1v32;
  return 0;
}

void
mg_destroy (Hierarchy *h)
{
  delete h;
}

/* smoothed-aggregation hierarchy of Z (level 0 borrows Z's device arrays) */
/* the Galerkin step of one level: R = P^T, A P (kept for the post
 * residual) and Ac = P^T (A P), symmetrised against rounding: every entry
 * (i, j) averaged with its mirror (j, i), found in row j's sorted columns
 * (the pattern of P^T A P is symmetric); the averages go to a copy so that
 * each pair reads the unsymmetrised values */
static void
galerkin (const HCsr &A, const HCsr &P, HCsr &R, HCsr &AP, HCsr &Ac)
{
  R = hcsr_transpose (P);
  AP = hcsr_gemm (A, P);
  Ac = hcsr_gemm (R, AP);
  decltype (Ac.v) vs (Ac.v.size ());
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < Ac.n; i++)
    for (int64_t k = Ac.rp[i]; k < Ac.rp[i + 1]; k++) {
      const int64_t j = Ac.ci[k];
      const int32_t *b = Ac.ci.data () + Ac.rp[j];
      const int32_t *e = Ac.ci.data () + Ac.rp[j + 1];
      const int32_t *f = std::lower_bound (b, e, (int32_t) i);
      const double mirror = (f != e && *f == i) ? Ac.v[Ac.rp[j] + (f - b)] : 0.;
      vs[k] = 0.5 * (Ac.v[k] + mirror);
    }
  Ac.v.swap (vs);
  Ac.m = Ac.n;
}

/* The first coarsening of a square host CSR on the host alone (no device
 * call): the level's lambda_max from the host CG-Lanczos, the smoothed
 * aggregation prolongator and the Galerkin step, with `threads` OpenMP
 * threads (0: the current default).  The set-up proper estimates
 * lambda_max on the device for large levels; this is for checking the host
 * products and their independence of the thread count. */
int
mg_host_galerkin (int64_t n, const int64_t *rowptr, const int32_t *colidx,
                  const double *vals, int threads, int64_t *nc_out,
                  int64_t *p_rowptr, int32_t *p_colidx, double *p_vals,
                  int64_t p_cap, int64_t *p_nnz, int64_t *c_rowptr,
                  int32_t *c_colidx, double *c_vals, int64_t c_cap,
                  int64_t *c_nnz)
{
  LGH_CHECK (n > 0 && rowptr && colidx && vals && nc_out && p_nnz && c_nnz,
             LGH_ERR_ARG_NULL, "mg_host_galerkin: null argument");
  LGH_CHECK (n < INT32_MAX, LGH_ERR_ARG_OUTOFRANGE,
             "mg_host_galerkin: n too large");
  LGH_CHECK (rowptr[0] == 0, LGH_ERR_ARG_WRONG,
             "mg_host_galerkin: rowptr[0] != 0");
  for (int64_t i = 0; i < n; i++)
    LGH_CHECK (rowptr[i + 1] >= rowptr[i], LGH_ERR_ARG_WRONG,
               "mg_host_galerkin: rowptr not monotone at row %lld",
               (long long) i);
  const int64_t nnz = rowptr[n];
  for (int64_t k = 0; k < nnz; k++)
    LGH_CHECK (colidx[k] >= 0 && colidx[k] < n, LGH_ERR_ARG_WRONG,
               "mg_host_galerkin: column out of range at entry %lld",
               (long long) k);
  HCsr A;
  A.n = A.m = n;
  A.rp.assign (rowptr, rowptr + n + 1);
  A.ci.resize (nnz);
  A.v.resize (nnz);
  memcpy (A.ci.data (), colidx, (size_t) nnz * sizeof (int32_t));
  memcpy (A.v.data (), vals, (size_t) nnz * sizeof (double));
  const int prev = omp_get_max_threads ();
  if (threads > 0) omp_set_num_threads (threads);
  const double lmax = lanczos_lmax (A, 40, 20260813ULL);
  HCsr P, R, AP, Ac;
  int64_t nc = 0;
  sa_coarsen (A, 0.0, lmax, P, nc);
  galerkin (A, P, R, AP, Ac);
  omp_set_num_threads (prev);
  *nc_out = nc;
  *p_nnz = P.rp[P.n];
  *c_nnz = Ac.rp[Ac.n];
  if (p_rowptr) {
    LGH_CHECK (p_cap >= *p_nnz && p_colidx && p_vals, LGH_ERR_ARG_OUTOFRANGE,
               "mg_host_galerkin: P needs %lld entries", (long long) *p_nnz);
    memcpy (p_rowptr, P.rp.data (), (size_t) (n + 1) * sizeof (int64_t));
    memcpy (p_colidx, P.ci.data (), (size_t) *p_nnz * sizeof (int32_t));
    memcpy (p_vals, P.v.data (), (size_t) *p_nnz * sizeof (double));
  }
  if (c_rowptr) {
    LGH_CHECK (c_cap >= *c_nnz && c_colidx && c_vals, LGH_ERR_ARG_OUTOFRANGE,
               "mg_host_galerkin: Ac needs %lld entries", (long long) *c_nnz);
    memcpy (c_rowptr, Ac.rp.data (), (size_t) (nc + 1) * sizeof (int64_t));
    memcpy (c_colidx, Ac.ci.data (), (size_t) *c_nnz * sizeof (int32_t));
    memcpy (c_vals, Ac.v.data (), (size_t) *c_nnz * sizeof (double));
  }
  return 0;
}

int
mg_build (const Csr &Z, int tile, double smoother_top, int nu, Hierarchy **out)
{
  (void) tile;
  const double t0 = wall ();
  /* phase seconds: download, Lanczos, coarsen, Galerkin products, uploads,
   * coarse inverse (printed to stderr when LGH_MG_VERBOSE is set) */
  double tp[6] = { 0., 0., 0., 0., 0., 0. };
  double tq = wall ();
  auto lap = [&] (int k) { const double t = wall (); tp[k] += t - tq; tq = t; };
  Hierarchy *h = new Hierarchy ();
  HCsr A;
  int rc = csr_download (Z, A);
  if (rc) { delete h; return rc; }
  lap (0);
  const int64_t coarse_max = 1500;
  const double theta = 0.0;
  for (int l = 0; l < 12; l++) {
    MgLevel lv;
    lv.n = A.n;
    lv.nu = nu > 0 ? nu : 2;
    if (l == 0) {
      lv.A = Z;
      lv.own = 0;
    } else {
      rc = csr_upload (A, lv.A);
      if (rc) { delete h; return rc; }
    }
    lap (4);
    /* the prolongator damping used the seed of level 0 on every level;
     * keep that estimate (identical on level 0, one Lanczos run fewer) */
    double lmax_own = 0.;
    if (A.n >= LZ_DEVICE_MIN) {
      rc = lanczos_lmax_dev (lv.A, 40, 20260813ULL + (uint64_t) l, &lv.smax);
      if (!rc && l > 0) rc = lanczos_lmax_dev (lv.A, 40, 20260813ULL, &lmax_own);
      if (rc) { delete h; return rc; }
    } else {
      lv.smax = lanczos_lmax (A, 40, 20260813ULL + (uint64_t) l);
      if (l > 0) lmax_own = lanczos_lmax (A, 40, 20260813ULL);
    }
    if (l == 0) lmax_own = lv.smax;
    lv.slo = 0.1 * lv.smax;
    lv.shi = smoother_top * lv.smax;
    if (lv.nu == 2 && !(A.n <= coarse_max || l == 11)) {
      rc = first_step_operator (lv);
      if (rc) { delete h; return rc; }
    }
    lap (1);
    if (A.n <= coarse_max || l == 11) {
      /* coarsest: dense inverse on the device, A^{-1} = L^{-T} L^{-1} */
      const int n0 = (int) A.n;
      std::vector<double> Dn ((size_t) n0 * n0, 0.);
      for (int64_t i = 0; i < A.n; i++)
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; k++)
          Dn[i + (size_t) A.ci[k] * n0] = A.v[k];
      h->n0 = n0;
      DBuf<double> G, G0, Li, work;
      DBuf<int> info;
      cudaStream_t s = stream ();
      rc = G.alloc ((size_t) n0 * n0);
      if (!rc) rc = G0.alloc ((size_t) n0 * n0);
      if (!rc) rc = Li.alloc ((size_t) n0 * n0);
      if (!rc) rc = info.alloc (4);
      if (!rc) rc = h->Ainv.alloc ((size_t) n0 * n0);
      if (!rc) rc = work.alloc (gemm_tn_work_elems (n0, n0, n0));
      if (!rc && cudaMemcpy (G.p, Dn.data (), Dn.size () * sizeof (double),
                             cudaMemcpyHostToDevice) != cudaSuccess)
        rc = set_error (LGH_ERR_GPU, "mg: coarse upload");
      if (!rc) rc = launch_potrf (n0, G.p, G0.p, 1, info.p, s);
      int hinfo[2] = { 0, 0 };
      if (!rc && cudaMemcpy (hinfo, info.p, 2 * sizeof (int),
                             cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = set_error (LGH_ERR_GPU, "mg: coarse info");
      if (!rc && hinfo[0]) rc = set_error (LGH_ERR_LIB, "mg: coarse operator not SPD");
      /* Li holds (L^{-1}) transposed: row-major view of L^{-1} */
      if (!rc) rc = launch_trtri_lower (n0, G.p, Li.p, 1, s);
      if (!rc) rc = launch_gemm_tn<double> (n0, n0, n0, Li.p, n0, Li.p, n0,
                                            h->Ainv.p, n0, 1, work.p, work.n, s);
      if (!rc && cudaStreamSynchronize (s) != cudaSuccess)
        rc = set_error (LGH_ERR_GPU, "mg: coarse inverse");
      if (rc) { delete h; return rc; }
      h->lev.push_back (lv);
      lv.own = 0;  /* ownership moved into h->lev */
      lap (5);
      break;
    }
    HCsr P;
    int64_t nc = 0;
    sa_coarsen (A, theta, lmax_own, P, nc);
    lap (2);
    if (nc >= A.n) {
      /* no coarsening progress: stop here with a dense coarse level is
       * impossible at this size */
      delete h;
      return set_error (LGH_ERR_SUP, "mg: aggregation made no progress at n=%lld",
                        (long long) A.n);
    }
    HCsr R, AP, Ac;
    galerkin (A, P, R, AP, Ac);
    lap (3);
    rc = csr_upload (P, lv.P);
    if (!rc) rc = csr_upload (R, lv.R);
    if (!rc && lv.f1v) rc = csr_upload (AP, lv.AP);
    if (rc) { delete h; return rc; }
    h->lev.push_back (lv);
    A = std::move (Ac);
    lap (4);
  }
  h->setup_s = wall () - t0;
  if (getenv ("LGH_MG_VERBOSE"))
    fprintf (stderr, "mg setup %.4f s: download %.4f lanczos %.4f coarsen %.4f "
             "galerkin %.4f upload %.4f coarse %.4f (levels %zu, coarse n %d)\n",
             h->setup_s, tp[0], tp[1], tp[2], tp[3], tp[4], tp[5],
             h->lev.size (), h->n0);
  *out = h;
  return 0;
}

/* ---- the block V-cycle ---------------------------------------------------- */

template <typename T>
static int
mg_work (Hierarchy *h, int ld, MgWork **w0, std::vector<MgWork> *own)
{
  std::vector<MgWork> &W = own ? *own
                           : (std::is_same<T, double>::value ? h->w64 : h->w32);
  if (W.size () != h->lev.size ()) W.resize (h->lev.size ());
  for (size_t l = 0; l < h->lev.size (); l++) {
    MgWork &w = W[l];
    if (w.cap >= ld) continue;
    const size_t bytes = (size_t) h->lev[l].n * ld * sizeof (T);
    if (l > 0) {   /* the finest level's B and X are the caller's */
      LGH_TRY (w.B.alloc (bytes));
      LGH_TRY (w.X.alloc (bytes));
    }
    /* the coarsest level solves densely from B into X; the two-step
     * smoother keeps no direction blocks (only other degrees use D0, D1) */
    if (l + 1 < h->lev.size ()) {
      LGH_TRY (w.R0.alloc (bytes));
      LGH_TRY (w.R1.alloc (bytes));
      if (h->lev[l].nu != 2) {
        LGH_TRY (w.D0.alloc (bytes));
        LGH_TRY (w.D1.alloc (bytes));
      }
    }
    w.cap = ld;
  }
  *w0 = W.data ();
  return 0;
}

template <typename T>
static const T *
zdinv_of (const Csr &A)
{
  if constexpr (std::is_same<T, double>::value) return A.dinv;
  else return A.dinv32;
}

/* the two-step Chebyshev-Jacobi coefficients on [slo, shi]: the first
 * step d = b1 D^{-1} r, the second d = a2 d + b2 D^{-1} r */
static void
cheb2_coeffs (const MgLevel &lv, double *b1, double *a2, double *b2)
{
  const double theta = 0.5 * (lv.shi + lv.slo);
  const double delta = 0.5 * (lv.shi - lv.slo);
  const double sigma1 = theta / delta;
  const double rho_old = 1.0 / sigma1;
  const double rho = 1.0 / (2.0 * sigma1 - rho_old);
  *b1 = 1.0 / theta;
  *a2 = rho * rho_old;
  *b2 = 2.0 * rho / delta;
}

/* Chebyshev-Jacobi smoothing in correction form on level l: R holds
 * B - A X on entry; nu terms; returns the buffer holding the residual */
template <typename T>
static int
mg_smooth (const MgLevel &lv, T *X, const T *B, T *R, T *Ra, T *D0, T *D1,
           int ld, bool pre, T **Rout, cudaStream_t s, KTrace *tr)
{
  /* pre: nu steps from X = 0 with the residual B (read, never written);
   * the residual after the last step is returned in *Rout.  post: from X
   * with the residual in R; the last step only updates X (its residual is
   * not needed), so it runs without the Z product.  Algorithmic bytes per
   * step: the operator (gather steps) plus the blocks each step reads and
   * writes. */
  const double sbase = (double) lv.A.nnz * (sizeof (T) + 4) + 8. * (lv.n + 1);
  const double sblk = (double) lv.n * ld * sizeof (T);
  const double theta = 0.5 * (lv.shi + lv.slo);
  const double delta = 0.5 * (lv.shi - lv.slo);
  const double sigma1 = theta / delta;
  double rho_old = 1.0 / sigma1;
  const T *Ro = pre ? B : R;
  T *Rn = pre ? R : Ra;
  T *Do = D0, *Dn = D1;
  if (lv.nu == 2) {
    /* the two-step polynomial in 6 block passes instead of 9: the first
     * step stores its residual alone, the second forms the first step's d
     * and x from that step's input residual (the same roundings, so the
     * same bits as two ordinary steps) */
    const double b1 = 1.0 / theta;
    const double rho = 1.0 / (2.0 * sigma1 - rho_old);
    const double a2 = rho * rho_old, b2 = 2.0 * rho / delta;
    const int f1 = CHEB_FIRST | CHEB_R_ONLY | (pre ? CHEB_ZERO_X : 0);
    if (lv.f1v && !pre) {
      /* post: both steps in one pass over r0 (gathered) and x; reads x
       * and r0, writes x (r1 stays in registers) */
      if (tr) LGH_TRY (tr->begin (K_MG_POST, sbase + 3. * sblk
                                  + (double) lv.n * sizeof (T), s));
      LGH_TRY (launch_spmm_cheb_post<T> (lv.F1, Ro, X, ld, ld,
                                         zdinv_of<T> (lv.A), a2,
                                         b2, b1, s));
      if (tr) LGH_TRY (tr->end (s));
      if (Rout) *Rout = nullptr;
      return 0;
    }
    if (lv.f1v) {
      /* r1 = r0 - (b1 Z D^{-1}) r0 with the products fl(b1 vd_ij) formed
       * once at set-up: the same products and order as the Chebyshev
       * kernel's first step, without its direction and x streams */
      if (tr) LGH_TRY (tr->begin (K_MG_FIRST, sbase + 2. * sblk, s));
      LGH_TRY (launch_spmm_mode<T> (lv.F1, Ro, ld, Rn, ld, ld, 2, Ro, ld, s));
      if (tr) LGH_TRY (tr->end (s));
    } else {
      if (tr) LGH_TRY (tr->begin (K_MG_SMOOTH, sbase + 2. * sblk, s));
      LGH_TRY (launch_cheb_step<T> (lv.A, X, Ro, Rn, nullptr, nullptr, ld, 0.,
                                    b1, f1, s));
      if (tr) LGH_TRY (tr->end (s));
    }
    T *R2 = (Rn == R) ? Ra : R;
    if (pre) {
      /* reads r1 (gathered), r0 = B (gathered); writes x, r2 */
      if (tr) LGH_TRY (tr->begin (K_MG_SMOOTH, sbase + 4. * sblk
                                  + (double) lv.n * sizeof (T), s));
      LGH_TRY (launch_cheb_step<T> (lv.A, X, Rn, R2, Ro, nullptr, ld, a2, b2,
                                    CHEB_PREV_R | CHEB_ZERO_X, s, b1));
      if (tr) LGH_TRY (tr->end (s));
      if (Rout) *Rout = R2;
    } else {
      /* reads x, r0, r1; writes x (no Z product) */
      if (tr) LGH_TRY (tr->begin (K_MG_TAIL, 4. * sblk
                                  + (double) lv.n * sizeof (T), s));
      LGH_TRY (launch_cheb_tail<T> (lv.A, X, Rn, Ro, ld, a2, b2, 0, s, b1));
      if (tr) LGH_TRY (tr->end (s));
      if (Rout) *Rout = nullptr;
    }
    return 0;
  }
  for (int k = 1; k <= lv.nu; k++) {
    double a, b;
    if (k == 1) { a = 0.; b = 1.0 / theta; }
    else {
      const double rho = 1.0 / (2.0 * sigma1 - rho_old);
      a = rho * rho_old;
      b = 2.0 * rho / delta;
      rho_old = rho;
    }
    const bool last = (k == lv.nu);
    if (!pre && last) {
      const double tb = (k == 1 ? 3. : 4.) * sblk + (double) lv.n * sizeof (T);
      if (tr) LGH_TRY (tr->begin (K_MG_TAIL, tb, s));
      LGH_TRY (launch_cheb_tail<T> (lv.A, X, Ro, Do, ld, a, b, k == 1, s));
      if (tr) LGH_TRY (tr->end (s));
      break;
    }
    const bool zx = pre && k == 1;
    const int flags = (k == 1 ? CHEB_FIRST : 0) | (zx ? CHEB_ZERO_X : 0)
                      | (last ? 0 : CHEB_STORE_D);
    const double nblk = 1. + (k == 1 ? 0. : 1.) + (zx ? 0. : 1.)   /* reads */
                        + 2. + (last ? 0. : 1.);                     /* writes */
    if (tr) LGH_TRY (tr->begin (K_MG_SMOOTH, sbase + nblk * sblk, s));
    LGH_TRY (launch_cheb_step<T> (lv.A, X, Ro, Rn, Do, Dn, ld, a, b, flags, s));
    if (tr) LGH_TRY (tr->end (s));
    Ro = Rn;
    Rn = (Rn == R) ? Ra : R;
    std::swap (Do, Dn);
  }
  if (Rout) *Rout = (T *) Ro;
  return 0;
}

template <typename T>
static int
vcycle_level (Hierarchy *h, MgWork *W, size_t l, const T *B, T *X, int ld,
              int w, cudaStream_t s, KTrace *trace)
{
  const MgLevel &lv = h->lev[l];
  const int64_t n = lv.n;
  KTrace *tr = (l == 0) ? trace : nullptr;   /* the fine level only */
  const double blk = (double) n * ld * sizeof (T);
  if (l + 1 == h->lev.size ()) {
    if (trace) LGH_TRY (trace->begin (K_MG_COARSE,
                                      (double) h->n0 * h->n0 * 8 + 2. * blk, s));
    LGH_TRY (launch_dense_apply<T> (h->n0, h->Ainv.p, B, X, w, ld, s));
    if (trace) LGH_TRY (trace->end (s));
    return 0;
  }
  MgWork &wk = W[l];
  T *R = (T *) wk.R0.p, *Ra = (T *) wk.R1.p;
  T *D0 = (T *) wk.D0.p, *D1 = (T *) wk.D1.p;
  /* pre-smoothing from X = 0 (the first step writes X without reading
   * it and reads the residual straight from B) */
  T *Rc = nullptr;
  LGH_TRY (mg_smooth<T> (lv, X, B, R, Ra, D0, D1, ld, true, &Rc, s, tr));
  /* restriction, coarse correction, prolongation */
  MgWork &wc = W[l + 1];
  T *Bc = (T *) wc.B.p, *Xc = (T *) wc.X.p;
  const double cblk = (double) h->lev[l + 1].n * ld * sizeof (T);
  if (tr) LGH_TRY (tr->begin (K_MG_RESTRICT, blk + cblk + 12. * lv.R.nnz, s));
  LGH_TRY (launch_spmm<T> (lv.R, Rc, ld, Bc, ld, ld, s));
  if (tr) LGH_TRY (tr->end (s));
  LGH_TRY (vcycle_level<T> (h, W, l + 1, Bc, Xc, ld, w, s, trace));
  constexpr int PW = Pack<T>::W;
  if (lv.nu == 2 && lv.f1v && lv.AP.n == n && Rc && ld <= 32 * 10 * PW) {
    /* r = r2 - (A P) xc: the residual of x + P xc from the pre-smoothing
     * residual r2 (the same value in exact arithmetic as B - A (x + P xc));
     * then the prolongation and both post-smoothing steps in one pass */
    T *Rp = (Rc == R) ? Ra : R;
    double b1, a2, b2;
    cheb2_coeffs (lv, &b1, &a2, &b2);
    if (tr) LGH_TRY (tr->begin (K_MG_RESID, 2. * blk + cblk
                                + (4. + sizeof (T)) * lv.AP.nnz, s));
    LGH_TRY (launch_spmm_mode<T> (lv.AP, Xc, ld, Rp, ld, ld, 2, Rc, ld, s));
    if (tr) LGH_TRY (tr->end (s));
    if (tr) LGH_TRY (tr->begin (K_MG_POSTP, 3. * blk + cblk + (double) n * sizeof (T)
                                + (4. + sizeof (T)) * (lv.F1.nnz + lv.P.nnz)
                                + 16. * (n + 1), s));
    LGH_TRY (launch_post_prolong<T> (lv.F1, lv.P, Rp, Xc, X, ld, ld,
                                     zdinv_of<T> (lv.A), a2, b2, b1, s));
    if (tr) LGH_TRY (tr->end (s));
    return 0;
  }
  if (tr) LGH_TRY (tr->begin (K_MG_PROLONG, 2. * blk + cblk + 12. * lv.P.nnz, s));
  LGH_TRY (launch_spmm_mode<T> (lv.P, Xc, ld, X, ld, ld, 1, nullptr, 0, s));
  if (tr) LGH_TRY (tr->end (s));
  /* post-smoothing: refresh the residual, then the same polynomial */
  if (tr) LGH_TRY (tr->begin (K_MG_RESID, 3. * blk + 12. * lv.A.nnz, s));
  LGH_TRY (launch_spmm_mode<T> (lv.A, X, ld, R, ld, ld, 2, B, ld, s));
  if (tr) LGH_TRY (tr->end (s));
  LGH_TRY (mg_smooth<T> (lv, X, nullptr, R, Ra, D0, D1, ld, false, nullptr, s,
                         tr));
  return 0;
}

template <typename T>
int
mg_vcycle (Hierarchy *h, const T *B, T *X, int ld, int w, cudaStream_t s,
           KTrace *tr, std::vector<MgWork> *work)
{
  MgWork *W;
  LGH_TRY (mg_work<T> (h, ld, &W, work));
  return vcycle_level<T> (h, W, 0, B, X, ld, w, s, tr);
}

template int mg_vcycle<double> (Hierarchy *, const double *, double *, int,
                                int, cudaStream_t, KTrace *,
                                std::vector<MgWork> *);
template int mg_vcycle<float> (Hierarchy *, const float *, float *, int, int,
                               cudaStream_t, KTrace *, std::vector<MgWork> *);

} /* namespace lgh */
