/* k_small.cu -- small dense FP64 linear algebra on the device (ell x ell,
 * column-major), replacing the reference's LAPACK calls:
 *
 *   potrf   DPOTRF("L") of the Gram matrix with the single diagonal jitter
 *           retry of glr_common_impl.h:386-398 (1e-12 tr/ell) or of
 *           glr_scalapack_impl.h:129-139 (1e-12 max(dmax, 1)).  One CTA,
 *           32-column panels staged in shared memory, right-looking.
 *   trtri   L^{-1} by column (one warp per column), optionally stored
 *           transposed so that X L^{-T} is a plain GEMM (the DTRSM of
 *           glr_common_impl.h:402).
 *   syev    DSYEVD("V","U") of the projected T (glr_common_impl.h:496-514):
 *           cyclic two-sided Jacobi in round-robin parallel order.  One
 *           cooperative launch; every CTA computes all rotations of a round
 *           from the same matrix (so all CTAs agree on convergence without
 *           communication), applies them to its slice of A and V, and meets
 *           the others at a bounded grid barrier.  Relative-accuracy
 *           rotation threshold, at most 40 sweeps.
 *   select  ordering by |lambda| descending, the cut max(trunc_abs,
 *           trunc_rel max|lambda|), treatment FLIP/RELU/NONE and the report
 *           fields (glr_common_impl.h:517-559; glr_scalapack_impl.h:375-425),
 *           plus the gathered eigenvector columns C_kept.
 */

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "lgh_device.cuh"
#include "lgh_internal.h"

namespace lgh
{

/* ---------------------------------------------------------------- potrf -- */

__global__ void __launch_bounds__ (1024)
k_potrf (int n, double *G, const double *G0, int jitter_mode, int *info,
         int nb)
{
  extern __shared__ double P[];     /* (n - k0) x (nb + 1) panel */
  __shared__ int fail;
  __shared__ double jit;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int ps = nb + 1;
  if (tid == 0) { info[0] = 0; info[1] = 0; }
  for (int attempt = 0; attempt < 2; attempt++) {
    if (attempt == 1) {
      /* re-form G (the factorization destroyed it) and jitter the diagonal */
      if (G0 == nullptr) break;
      for (int e = tid; e < n * n; e += nt) G[e] = G0[e];
      __syncthreads ();
      if (tid == 0) {
        double v = 0.;
        if (jitter_mode == 0) {
          for (int i = 0; i < n; i++) v += G[i + (size_t) i * n];
          v = 1e-12 * v / n;
        } else {
          for (int i = 0; i < n; i++) v = fmax (v, G[i + (size_t) i * n]);
          v = 1e-12 * fmax (v, 1.0);
        }
        jit = v;
        info[1] = 1;
      }
      __syncthreads ();
      for (int i = tid; i < n; i += nt) G[i + (size_t) i * n] += jit;
      __syncthreads ();
    }
    if (tid == 0) fail = 0;
    __syncthreads ();
    for (int k0 = 0; k0 < n && !fail; k0 += nb) {
      const int kb = min (nb, n - k0);
      const int m = n - k0;
      for (int e = tid; e < m * kb; e += nt) {
        const int r = e % m, kk = e / m;
        P[r * ps + kk] = G[(k0 + r) + (size_t) (k0 + kk) * n];
      }
      __syncthreads ();
      for (int kk = 0; kk < kb; kk++) {
        if (tid == 0) {
          const double d = P[kk * ps + kk];
          if (!(d > 0.) || !isfinite (d)) fail = 1;
          else P[kk * ps + kk] = sqrt (d);
        }
        __syncthreads ();
        if (fail) break;
        const double dk = P[kk * ps + kk];
        for (int r = kk + 1 + tid; r < m; r += nt) P[r * ps + kk] /= dk;
        __syncthreads ();
        const int rem = kb - kk - 1;
        for (int e = tid; e < m * rem; e += nt) {
          const int r = e % m, jj = kk + 1 + e / m;
          if (r >= jj) P[r * ps + jj] -= P[r * ps + kk] * P[jj * ps + kk];
        }
        __syncthreads ();
      }
      if (fail) break;
      for (int e = tid; e < m * kb; e += nt) {
        const int r = e % m, kk = e / m;
        if (r >= kk) G[(k0 + r) + (size_t) (k0 + kk) * n] = P[r * ps + kk];
      }
      /* trailing update G(i, j) -= P(i, :) P(j, :)^T, i >= j >= k0 + kb */
      const int mt = m - kb;
      for (int e = tid; e < mt * mt; e += nt) {
        const int ii = e % mt, jj = e / mt;
        if (ii < jj) continue;
        const int ri = kb + ii, rj = kb + jj;
        double s = 0.;
        for (int kk = 0; kk < kb; kk++) s = fma (P[ri * ps + kk], P[rj * ps + kk], s);
        G[(k0 + ri) + (size_t) (k0 + rj) * n] -= s;
      }
      __syncthreads ();
    }
    __syncthreads ();
    if (!fail) break;
  }
  __syncthreads ();
  if (tid == 0 && fail) info[0] = 1;
  /* clear the strict upper triangle */
  for (int e = tid; e < n * n; e += nt) {
    const int i = e % n, j = e / n;
    if (i < j) G[e] = 0.;
  }
}

int
launch_potrf (int n, double *G, double *G0, int jitter_mode, int *info,
              cudaStream_t s)
{
  if (n <= 0) return 0;
  const int nb = (n <= 800) ? 32 : 16;
  const int smem = n * (nb + 1) * (int) sizeof (double);
  LGH_CHECK (smem <= 220 * 1024, LGH_ERR_SUP, "potrf: n=%d too large", n);
  if (G0) LGH_CUDA (cudaMemcpyAsync (G0, G, (size_t) n * n * sizeof (double),
                                     cudaMemcpyDeviceToDevice, s));
  LGH_CUDA (cudaFuncSetAttribute (k_potrf,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem));
  k_potrf<<<1, 1024, smem, s>>> (n, G, G0, jitter_mode, info, nb);
  LGH_LAUNCH_CHECK ();
  return 0;
}

/* ---------------------------------------------------------------- trtri -- */

__global__ void __launch_bounds__ (256)
k_trtri_lower (int n, const double *__restrict__ L, double *__restrict__ out,
               int transpose)
{
  extern __shared__ double xs[];    /* 8 warps x n */
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * 8 + warp;
  if (j >= n) return;
  double *x = xs + (size_t) warp * n;
  for (int i = lane; i < n; i += 32) x[i] = (i == j) ? 1. : 0.;
  __syncwarp ();
  for (int k = j; k < n; k++) {
    const double xk = x[k] / L[k + (size_t) k * n];
    __syncwarp ();
    if (lane == 0) x[k] = xk;
    for (int i = k + 1 + lane; i < n; i += 32) x[i] -= L[i + (size_t) k * n] * xk;
    __syncwarp ();
  }
  for (int i = lane; i < n; i += 32) {
    const double v = (i >= j) ? x[i] : 0.;
    if (transpose) out[j + (size_t) i * n] = v;
    else out[i + (size_t) j * n] = v;
  }
}

int
launch_trtri_lower (int n, const double *L, double *Linv, int transpose,
                    cudaStream_t s)
{
  if (n <= 0) return 0;
  const int smem = 8 * n * (int) sizeof (double);
  LGH_CUDA (cudaFuncSetAttribute (k_trtri_lower,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem));
  k_trtri_lower<<<(n + 7) / 8, 256, smem, s>>> (n, L, Linv, transpose);
  LGH_LAUNCH_CHECK ();
  return 0;
}

/* ------------------------------------------------------------- jacobi -- */

struct JacobiCtl
{
  unsigned count, gen;
  int err, sweeps;
};

/* index at position `pos` in round r of the round-robin over np entries */
__device__ __forceinline__ int
rr_index (int pos, int r, int np)
{
  return pos == 0 ? 0 : 1 + ((pos - 1 + r) % (np - 1));
}

__global__ void __launch_bounds__ (256)
k_jacobi (int n, int np, double *A, double *A2, double *V, double *V2,
          JacobiCtl *ctl, int max_sweeps)
{
  extern __shared__ double sh[];
  const int npair = np / 2;
  double *cs = sh;                  /* c per pair    */
  double *sn = cs + npair;          /* s per pair    */
  double *tt = sn + npair;          /* t per pair    */
  int *pp = (int *) (tt + npair);   /* p per pair    */
  int *qq = pp + npair;             /* q per pair    */
  int *pr = qq + npair;             /* pair of index */
  __shared__ int any_rot;
  const int64_t nn = (int64_t) n * n;
  const int64_t gtid = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t) gridDim.x * blockDim.x;
  /* V = I */
  for (int64_t e = gtid; e < nn; e += gstride)
    V[e] = ((e % n) == (e / n)) ? 1. : 0.;
  if (!grid_barrier (&ctl->count, &ctl->gen, &ctl->err)) return;
  int done = 0;
  for (int sweep = 0; sweep < max_sweeps; sweep++) {
    if (threadIdx.x == 0) any_rot = 0;
    __syncthreads ();
    for (int r = 0; r < np - 1; r++) {
      for (int k = threadIdx.x; k < npair; k += blockDim.x) {
        int p = rr_index (k, r, np), q = rr_index (np - 1 - k, r, np);
        if (p > q) { int t = p; p = q; q = t; }
        double c = 1., s = 0., t = 0.;
        if (q < n) {
          const double apq = A[p + (size_t) q * n];
          const double app = A[p + (size_t) p * n];
          const double aqq = A[q + (size_t) q * n];
          if (fabs (apq) > 1e-300
              && fabs (apq) > 1e-15 * sqrt (fabs (app) * fabs (aqq))) {
            const double th = (aqq - app) / (2. * apq);
            t = (th >= 0. ? 1. : -1.) / (fabs (th) + sqrt (1. + th * th));
            c = 1. / sqrt (1. + t * t);
            s = t * c;
            any_rot = 1;
          }
        }
        cs[k] = c; sn[k] = s; tt[k] = t; pp[k] = p; qq[k] = q;
        if (p < np) pr[p] = k;
        if (q < np) pr[q] = k;
      }
      __syncthreads ();
      for (int64_t e = gtid; e < nn; e += gstride) {
        const int i = (int) (e % n), j = (int) (e / n);
        const int ki = pr[i], kj = pr[j];
        /* a pair with the padding index (odd n) never rotates: clamp its
         * partner to itself so every load stays inside the n x n matrix */
        const int pi = pp[ki], pj = pp[kj];
        const int qi = (qq[ki] < n) ? qq[ki] : pi;
        const int qj = (qq[kj] < n) ? qq[kj] : pj;
        double v;
        if (ki == kj && i != j) {
          /* the annihilated pair (kept as is when the rotation was skipped) */
          v = (sn[ki] != 0.) ? 0. : A[e];
        } else if (ki == kj) {
          const double apq = A[pi + (size_t) qi * n];
          v = (i == pi) ? A[i + (size_t) i * n] - tt[ki] * apq
                        : A[i + (size_t) i * n] + tt[ki] * apq;
        } else {
          /* weights of rows/cols: index == p -> (c, -s); == q -> (s, c) */
          const double ci = cs[ki], si = sn[ki], cj = cs[kj], sj = sn[kj];
          const double wi0 = (i == pi) ? ci : si, wi1 = (i == pi) ? -si : ci;
          const double wj0 = (j == pj) ? cj : sj, wj1 = (j == pj) ? -sj : cj;
          const double a00 = A[pi + (size_t) pj * n], a01 = A[pi + (size_t) qj * n];
          const double a10 = A[qi + (size_t) pj * n], a11 = A[qi + (size_t) qj * n];
          v = wi0 * (a00 * wj0 + a01 * wj1) + wi1 * (a10 * wj0 + a11 * wj1);
        }
        A2[e] = v;
        /* V' = V J : column j mixes V(:, pj), V(:, qj) */
        {
          const double cj = cs[kj], sj = sn[kj];
          const double wj0 = (j == pj) ? cj : sj, wj1 = (j == pj) ? -sj : cj;
          V2[e] = V[i + (size_t) pj * n] * wj0 + V[i + (size_t) qj * n] * wj1;
        }
      }
      if (!grid_barrier (&ctl->count, &ctl->gen, &ctl->err)) return;
      { double *t = A; A = A2; A2 = t; }
      { double *t = V; V = V2; V2 = t; }
    }
    __syncthreads ();
    done++;
    if (!any_rot) break;
  }
  /* the result sits in whichever buffers the last round wrote; the host
   * locates it from the number of completed sweeps */
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->sweeps = done;
}

__global__ void
k_jacobi_finish (int n, const double *A, const double *V, double *Vout,
                 double *w)
{
  const int64_t nn = (int64_t) n * n;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < nn;
       e += (int64_t) gridDim.x * blockDim.x) {
    if (Vout != V) Vout[e] = V[e];
    const int i = (int) (e % n), j = (int) (e / n);
    if (i == j) w[i] = A[e];
  }
}

int
launch_syev_jacobi (int n, double *A, double *V, double *w, double *A2,
                    double *V2, int *sweeps, cudaStream_t s)
{
  if (n <= 0) return 0;
  LGH_CHECK (n <= 2048, LGH_ERR_SUP, "syev: n=%d > 2048", n);
  if (n == 1) {
    LGH_CUDA (cudaMemcpyAsync (w, A, sizeof (double), cudaMemcpyDeviceToDevice, s));
    double one = 1.;
    LGH_CUDA (cudaMemcpyAsync (V, &one, sizeof (double), cudaMemcpyHostToDevice, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    if (sweeps) *sweeps = 0;
    return 0;
  }
  const int np = n + (n & 1);
  const int npair = np / 2;
  const int smem = npair * 3 * (int) sizeof (double) + (2 * npair + np) * (int) sizeof (int);
  LGH_CUDA (cudaFuncSetAttribute (k_jacobi,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem));
  int per_sm = 0;
  LGH_CUDA (cudaOccupancyMaxActiveBlocksPerMultiprocessor (&per_sm, k_jacobi,
                                                           256, smem));
  LGH_CHECK (per_sm >= 1, LGH_ERR_GPU, "syev: kernel cannot be resident");
  /* two CTAs per SM (within what is resident, as the cooperative launch
   * needs): a round's element updates are the larger part of its time, so
   * more CTAs shorten it despite the wider barrier (measured at n = 220:
   * 15.7 ms on 48 CTAs, 11.6 ms on 296; at n = 520: 65 ms on 148 CTAs,
   * 51 ms on 296); the result does not depend on the grid.  Small
   * problems keep about one CTA per 128 matrix entries (n = 220 still
   * gets 296), so that a 10 x 10 eigensolve does not pay a 296-CTA
   * barrier every round. */
  const int64_t by_size = std::max<int64_t> (1, ((int64_t) n * n + 127) / 128);
  int grid = (int) std::min<int64_t> (std::min<int64_t> (2 * (int64_t) num_sms (),
                                                         (int64_t) num_sms () * per_sm),
                                      by_size);
  JacobiCtl *ctl;
  LGH_TRY (dalloc ((void **) &ctl, sizeof (JacobiCtl)));
  cudaMemsetAsync (ctl, 0, sizeof (JacobiCtl), s);
  int max_sweeps = 40;
  void *args[] = { &n, (void *) &np, &A, &A2, &V, &V2, &ctl, &max_sweeps };
  cudaError_t e = cudaLaunchCooperativeKernel ((const void *) k_jacobi, grid,
                                               256, args, smem, s);
  if (e != cudaSuccess) {
    dfree (ctl);
    return set_error (LGH_ERR_GPU, "syev: cooperative launch: %s",
                      cudaGetErrorString (e));
  }
  JacobiCtl h;
  e = cudaMemcpyAsync (&h, ctl, sizeof (JacobiCtl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize (s);
  dfree (ctl);
  if (e != cudaSuccess)
    return set_error (LGH_ERR_GPU, "syev: %s", cudaGetErrorString (e));
  LGH_CHECK (h.err == 0, LGH_ERR_GPU, "syev: grid barrier timed out");
  /* rounds per sweep = np - 1; each round swaps the buffers */
  const long swaps = (long) h.sweeps * (np - 1);
  const double *Af = (swaps & 1) ? A2 : A;
  const double *Vf = (swaps & 1) ? V2 : V;
  k_jacobi_finish<<<std::max (1, std::min (num_sms () * 4, (n * n + 255) / 256)),
                    256, 0, s>>> (n, Af, Vf, V, w);
  LGH_LAUNCH_CHECK ();
  if (sweeps) *sweeps = h.sweeps;
  return 0;
}

/* ------------------------------------------------------------- select -- */

__global__ void __launch_bounds__ (1024)
k_select (int n, const double *__restrict__ w, const double *__restrict__ V,
          double trunc_abs, double trunc_rel, int treat, int *order,
          double *sel, double *lam, double *C)
{
  __shared__ double absmax, cut;
  __shared__ int kept;
  const int tid = threadIdx.x, nt = blockDim.x;
  /* rank: |w| descending, ties by larger raw value, then by index */
  for (int i = tid; i < n; i += nt) {
    const double ai = fabs (w[i]);
    int rank = 0;
    for (int j = 0; j < n; j++) {
      const double aj = fabs (w[j]);
      if (aj > ai || (aj == ai && (w[j] > w[i] || (w[j] == w[i] && j < i))))
        rank++;
    }
    order[rank] = i;
  }
  __syncthreads ();
  if (tid == 0) {
    absmax = fabs (w[order[0]]);
    double c = 0.;
    if (trunc_abs > 0.) c = fmax (c, trunc_abs);
    if (trunc_rel > 0.) c = fmax (c, trunc_rel * absmax);
    cut = c;
    int k = 0;
    while (k < n && fabs (w[order[k]]) > c) k++;
    kept = k;
    double mn = w[0], mx = w[0];
    int nneg = 0;
    for (int i = 0; i < n; i++) {
      mn = fmin (mn, w[i]);
      mx = fmax (mx, w[i]);
      if (w[i] < 0.) nneg++;
    }
    sel[0] = k;
    sel[1] = absmax;
    sel[2] = (k < n) ? fabs (w[order[k]]) : 0.;
    sel[3] = mn;
    sel[4] = mx;
    sel[5] = nneg;
  }
  __syncthreads ();
  for (int j = tid; j < kept; j += nt) {
    const double l = w[order[j]];
    lam[j] = (treat == 0) ? fabs (l) : (treat == 1 ? fmax (l, 0.) : l);
  }
  for (int64_t e = tid; e < (int64_t) n * kept; e += nt) {
    const int i = (int) (e % n), j = (int) (e / n);
    C[e] = V[i + (size_t) order[j] * n];
  }
}

int
launch_select (int n, const double *w, const double *V, double trunc_abs,
               double trunc_rel, int treat, int *order, double *sel,
               double *lam, double *C, cudaStream_t s)
{
  k_select<<<1, 1024, 0, s>>> (n, w, V, trunc_abs, trunc_rel, treat, order,
                               sel, lam, C);
  LGH_LAUNCH_CHECK ();
  return 0;
}

/* extreme eigenvalues of the CG-Lanczos tridiagonal T(k,k) = 1/a_k +
 * b_{k-1}/a_{k-1}, T(k,k+1) = sqrt(b_k)/a_k, through the device Jacobi */
int
device_tridiag_extremes (int m, const double *alpha, const double *beta,
                         double *emin, double *emax)
{
  cudaStream_t s = stream ();
  std::vector<double> T ((size_t) m * m, 0.);
  for (int k = 0; k < m; k++) {
    double d = 1. / alpha[k];
    if (k > 0) d += beta[k - 1] / alpha[k - 1];
    T[k + (size_t) k * m] = d;
    if (k + 1 < m) {
      const double e = sqrt (fabs (beta[k])) / alpha[k];
      T[k + (size_t) (k + 1) * m] = e;
      T[k + 1 + (size_t) k * m] = e;
    }
  }
  DBuf<double> A, A2, V, V2, w;
  LGH_TRY (A.alloc ((size_t) m * m));
  LGH_TRY (A2.alloc ((size_t) m * m));
  LGH_TRY (V.alloc ((size_t) m * m));
  LGH_TRY (V2.alloc ((size_t) m * m));
  LGH_TRY (w.alloc (m));
  LGH_CUDA (cudaMemcpyAsync (A.p, T.data (), T.size () * sizeof (double),
                             cudaMemcpyHostToDevice, s));
  LGH_TRY (launch_syev_jacobi (m, A.p, V.p, w.p, A2.p, V2.p, nullptr, s));
  std::vector<double> wh (m);
  LGH_CUDA (cudaMemcpyAsync (wh.data (), w.p, m * sizeof (double),
                             cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  *emin = *std::min_element (wh.begin (), wh.end ());
  *emax = *std::max_element (wh.begin (), wh.end ());
  return 0;
}

} /* namespace lgh */
