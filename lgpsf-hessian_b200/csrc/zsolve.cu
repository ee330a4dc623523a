/* zsolve.cu -- blocked Z-solves on row-major blocks.
 *
 * Restates the reference's Z-solve contract (include/lgpsf_hessian/impl/
 * zsolve_impl.h) for one device:
 *   mode 0/1  per-column preconditioned CG (the semantics of the per-column
 *             KSPSolve of zsolve_impl.h:674-715: CG, zero initial guess,
 *             preconditioned-residual norm, rtol = ksp_rtol, 10000-iteration
 *             cap), run for all columns of a block at once with per-column
 *             alpha/beta and a per-column convergence mask;
 *   mode 2    fixed-count Chebyshev (zsolve_impl.h:94-141), nit from the
 *             margined spectral interval.
 * The preconditioner is Jacobi (the reference's PCGAMG is replaced; the
 * aggregation V-cycle of mode 3 lives in mg.cu).
 *
 * Each CG iteration is two fused kernels:
 *   k_pcg_pq   p_new = D^{-1} r + beta p_old, computed on the fly at every
 *              neighbour row, q = Z p_new, and the per-column dot (p, q);
 *              the last CTA (atomic ticket) reduces the per-CTA partials in
 *              a fixed order and sets alpha = (r, z) / (p, q).
 *   k_pcg_upd  x += alpha p, r -= alpha q, z = D^{-1} r, dots (r, z) and
 *              (z, z); the last CTA sets beta, the convergence mask and the
 *              count of active columns.
 * HBM traffic per iteration: 10 N w s (Chebyshev: 6 N w s, one kernel).
 * Every reduction is deterministic: reruns are bitwise identical and a
 * column's result does not depend on the other columns of the block.
 */

#include <algorithm>
#include <cmath>
#include <mutex>
#include <type_traits>
#include <unordered_map>

#include "lgh_device.cuh"
#include "lgh_internal.h"
#include "lgh_ktime.h"
#include "lgh_mg.h"

namespace lgh
{

int row_grid (int64_t n, int glog);

constexpr int ZS_THREADS = 256;
constexpr int ZS_MAXCH = 8;

/* per-column scalar slots in ZWork::scal (each `cap` long) */
enum { S_RZ = 0, S_ALPHA, S_BETA, S_NORM0, S_NSLOT };
/* int slots in ZWork::ival */
enum { I_ACTIVE = 0, I_ITS, I_NSLOT };

struct ZK
{
  int64_t n;
  const int64_t *rowptr;
  const int32_t *col;
};

#define ZS_GROUP_SETUP()                                                     \
  constexpr int W = Pack<T>::W;                                              \
  const int G = 1 << glog;                                                   \
  const int lane = threadIdx.x & (G - 1);                                    \
  const int group = threadIdx.x >> glog;                                     \
  const int ngroups = blockDim.x >> glog;                                    \
  const unsigned gmask = (G == 32) ? 0xffffffffu                             \
      : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));               \
  (void) gmask;                                                              \
  /* row tiles of ngroups rows interleaved over the CTAs: the resident   \
   * CTAs sweep one narrow band, so stencil neighbours hit in L2 */      \
  

/* ---- init: R = S B (pads zero), X = 0, P = 0; rz, norm0, mask ---------- */
template <typename T, int CH>
__global__ void __launch_bounds__ (ZS_THREADS, (CH * (16 / sizeof (T)) <= 8 ? 3 : 2))
k_pcg_init (ZK z, const T *__restrict__ dinv, const T *__restrict__ Bsrc,
            int ldb, const double *__restrict__ rs_in, T *X, T *R, T *P,
            int ld, int nvec, int glog, int w, double *partA, double *partB,
            unsigned *counter, double *scal, int *ival, int cap)
{
  extern __shared__ double red[];
  ZS_GROUP_SETUP ();
  double aRZ[CH][W], aZZ[CH][W];
#pragma unroll
  for (int h = 0; h < CH; h++)
#pragma unroll
    for (int e = 0; e < W; e++) { aRZ[h][e] = 0.; aZZ[h][e] = 0.; }
  for (int64_t i = (int64_t) blockIdx.x * ngroups + group; i < z.n;
       i += (int64_t) gridDim.x * ngroups) {
    const double sc = rs_in ? rs_in[i] : 1.0;
    const double di = (double) dinv[i];
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        Pack<T> r;
#pragma unroll
        for (int e = 0; e < W; e++) {
          /* scalar loads guarded by c < w: the source may be a single
           * vector (ldb = 1) or an unaligned view */
          const int c = vi * W + e;
          const T bv = (c < w) ? (T) (sc * (double) Bsrc[i * ldb + c]) : T (0);
          r.v[e] = bv;
          const double zz = di * (double) bv;
          aRZ[h][e] += (double) bv * zz;
          aZZ[h][e] += zz * zz;
        }
        stp (R + i * ld + vi * W, r);
        stp (X + i * ld + vi * W, pzero<T> ());
        stp (P + i * ld + vi * W, pzero<T> ());
      }
    }
  }
  block_colsum_store<T, CH> (aRZ, lane, group, G, nvec, ld, red, partA);
  block_colsum_store<T, CH> (aZZ, lane, group, G, nvec, ld, red, partB);
  double *rz = scal + S_RZ * cap, *al = scal + S_ALPHA * cap;
  double *be = scal + S_BETA * cap, *n0 = scal + S_NORM0 * cap;
  int *act = ival + I_ACTIVE * cap, *its = ival + I_ITS * cap;
  bool last = last_block_reduce2 (partA, partB, ld, counter,
      [&] (int c, double srz, double szz) {
        rz[c] = srz;
        n0[c] = sqrt (szz);
        act[c] = (c < w && szz > 0.) ? 1 : 0;
        al[c] = 0.;
        be[c] = 0.;
        its[c] = 0;
      });
  if (last) {
    __syncthreads ();
    if (threadIdx.x == 0) {
      int cnt = 0;
      for (int c = 0; c < ld; c++) cnt += act[c];
      ival[I_NSLOT * cap] = cnt;
    }
  }
}

/* ---- p_new on the fly, q = Z p_new, alpha ------------------------------- */
template <typename T, int CH>
__global__ void __launch_bounds__ (ZS_THREADS, (CH * (16 / sizeof (T)) <= 8 ? 3 : 2))
k_pcg_pq (ZK z, const T *__restrict__ vals, const T *__restrict__ dinv,
          const T *__restrict__ R, const T *__restrict__ Pold,
          T *__restrict__ Pnew, T *__restrict__ Qv, int ld, int nvec,
          int glog, int first, double *partA, unsigned *counter,
          double *scal, int *ival, int cap)
{
  extern __shared__ double red[];
  ZS_GROUP_SETUP ();
  const double *beta = scal + S_BETA * cap;
  T bet[CH][W];
#pragma unroll
  for (int h = 0; h < CH; h++)
#pragma unroll
    for (int e = 0; e < W; e++) {
      const int c = (lane + h * G) * W + e;
      bet[h][e] = (!first && c < ld) ? (T) beta[c] : T (0);
    }
  double aPQ[CH][W];
#pragma unroll
  for (int h = 0; h < CH; h++)
#pragma unroll
    for (int e = 0; e < W; e++) aPQ[h][e] = 0.;
  for (int64_t i = (int64_t) blockIdx.x * ngroups + group; i < z.n;
       i += (int64_t) gridDim.x * ngroups) {
    T acc[CH][W];
#pragma unroll
    for (int h = 0; h < CH; h++)
#pragma unroll
      for (int e = 0; e < W; e++) acc[h][e] = T (0);
    const int64_t k0 = z.rowptr[i], k1 = z.rowptr[i + 1];
    for (int64_t kb = k0; kb < k1; kb += G) {
      const int cnt = (int) ((k1 - kb) < G ? (k1 - kb) : G);
      int mc = 0;
      T mv = T (0), md = T (0);
      if (lane < cnt) {
        mc = z.col[kb + lane];
        mv = vals[kb + lane];
        md = dinv[mc];
      }
      for (int t = 0; t < cnt; t++) {
        const int c = __shfl_sync (gmask, mc, t, G);
        const T v = __shfl_sync (gmask, mv, t, G);
        const T dj = __shfl_sync (gmask, md, t, G);
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = lane + h * G;
          if (vi < nvec) {
            Pack<T> rj = ldp (R + (int64_t) c * ld + vi * W);
            Pack<T> pj = first ? pzero<T> () : ldp (Pold + (int64_t) c * ld + vi * W);
#pragma unroll
            for (int e = 0; e < W; e++)
              acc[h][e] = fma (v, fma (dj, rj.v[e], bet[h][e] * pj.v[e]),
                               acc[h][e]);
          }
        }
      }
    }
    const T di = dinv[i];
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        Pack<T> ri = ldp (R + i * ld + vi * W);
        Pack<T> pi = first ? pzero<T> () : ldp (Pold + i * ld + vi * W);
        Pack<T> pn, q;
#pragma unroll
        for (int e = 0; e < W; e++) {
          pn.v[e] = fma (di, ri.v[e], bet[h][e] * pi.v[e]);
          q.v[e] = acc[h][e];
          aPQ[h][e] += (double) pn.v[e] * (double) q.v[e];
        }
        stp (Pnew + i * ld + vi * W, pn);
        stp (Qv + i * ld + vi * W, q);
      }
    }
  }
  block_colsum_store<T, CH> (aPQ, lane, group, G, nvec, ld, red, partA);
  const double *rz = scal + S_RZ * cap;
  double *al = scal + S_ALPHA * cap;
  int *act = ival + I_ACTIVE * cap;
  last_block_reduce (partA, ld, counter, [&] (int c, double pq) {
    if (act[c]) {
      if (pq != 0. && isfinite (pq)) al[c] = rz[c] / pq;
      else { al[c] = 0.; act[c] = 0; }
    } else {
      al[c] = 0.;
    }
  });
}

/* ---- x += alpha p, r -= alpha q, dots, beta, convergence ---------------- */
template <typename T, int CH>
__global__ void __launch_bounds__ (ZS_THREADS, (CH * (16 / sizeof (T)) <= 8 ? 3 : 2))
k_pcg_upd (ZK z, const T *__restrict__ dinv, T *__restrict__ X,
           T *__restrict__ R,
           const T *__restrict__ Pn, const T *__restrict__ Qv, int ld,
           int nvec, int glog, double *partA, double *partB,
           unsigned *counter, double *scal, int *ival, int cap, double rtol,
           int iter, double *hist)
{
  extern __shared__ double red[];
  ZS_GROUP_SETUP ();
  const double *alpha = scal + S_ALPHA * cap;
  T al[CH][W];
#pragma unroll
  for (int h = 0; h < CH; h++)
#pragma unroll
    for (int e = 0; e < W; e++) {
      const int c = (lane + h * G) * W + e;
      al[h][e] = (c < ld) ? (T) alpha[c] : T (0);
    }
  double aRZ[CH][W], aZZ[CH][W];
#pragma unroll
  for (int h = 0; h < CH; h++)
#pragma unroll
    for (int e = 0; e < W; e++) { aRZ[h][e] = 0.; aZZ[h][e] = 0.; }
  for (int64_t i = (int64_t) blockIdx.x * ngroups + group; i < z.n;
       i += (int64_t) gridDim.x * ngroups) {
    const T di = dinv[i];
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        const int64_t o = i * ld + vi * W;
        Pack<T> x = ldp (X + o), r = ldp (R + o), p = ldp (Pn + o),
                q = ldp (Qv + o);
#pragma unroll
        for (int e = 0; e < W; e++) {
          x.v[e] = fma (al[h][e], p.v[e], x.v[e]);
          r.v[e] = fma (-al[h][e], q.v[e], r.v[e]);
          const double zz = (double) di * (double) r.v[e];
          aRZ[h][e] += (double) r.v[e] * zz;
          aZZ[h][e] += zz * zz;
        }
        stp (X + o, x);
        stp (R + o, r);
      }
    }
  }
  block_colsum_store<T, CH> (aRZ, lane, group, G, nvec, ld, red, partA);
  block_colsum_store<T, CH> (aZZ, lane, group, G, nvec, ld, red, partB);
  double *rz = scal + S_RZ * cap, *be = scal + S_BETA * cap;
  double *al_g = scal + S_ALPHA * cap;
  const double *n0 = scal + S_NORM0 * cap;
  int *act = ival + I_ACTIVE * cap, *its = ival + I_ITS * cap;
  bool last = last_block_reduce2 (partA, partB, ld, counter,
      [&] (int c, double srz, double szz) {
        if (!act[c]) { be[c] = 0.; return; }
        const double b = (rz[c] != 0.) ? srz / rz[c] : 0.;
        if (hist != nullptr && c == 0 && iter < 10000) {
          hist[2 * iter] = al_g[0];
          hist[2 * iter + 1] = b;
        }
        rz[c] = srz;
        be[c] = b;
        if (sqrt (szz) <= rtol * n0[c] || srz == 0.) {
          act[c] = 0;
          be[c] = 0.;
          al_g[c] = 0.;
          its[c] = iter + 1;
        }
      });
  if (last) {
    __syncthreads ();
    if (threadIdx.x == 0) {
      int cnt = 0;
      for (int c = 0; c < ld; c++) cnt += act[c];
      ival[I_NSLOT * cap] = cnt;
    }
  }
}

/* ---- Chebyshev: d_new = a d + b D^{-1} r (on the fly at neighbours),
 *      x += d_new, r_new = r - Z d_new (zsolve_impl.h:108-141) ----------- */
template <typename T, int CH, bool PR = false>
__global__ void __launch_bounds__ (ZS_THREADS, (CH * (16 / sizeof (T)) <= 8 ? 4 : 2))
k_cheb (ZK z, const T *__restrict__ vals, const T *__restrict__ vdv,
        const T *__restrict__ dinv, T *__restrict__ X,
        const T *__restrict__ Rold, T *__restrict__ Rnew,
        const T *__restrict__ Dold, T *__restrict__ Dnew, int ld, int nvec,
        int glog, T a, T b, int flags, T bp)
{
  /* PR: the previous step was a first step (d = bp D^{-1} r_prev) that
   * stored only its residual; Dold then holds r_prev, and the previous d
   * and x are formed here with that step's roundings: d_prev = (bp
   * dinv_j) r_prev_j at every neighbour and at the row, x_prev = d_prev
   * (from x = 0) or x + d_prev.  CHEB_R_ONLY: store the new residual
   * alone (the next step forms d and x the same way). */
  /* r_new = r - Z d_new with d_new = a d + b D^{-1} r formed at each
   * neighbour: sum_j (b vd_ij r_j + a v_ij d_j), vd_ij = v_ij / z_jj.
   * Software pipeline over the group's rows: the next row's bounds and
   * its first G (column, value, value/diagonal) triples are loaded while
   * the current row's neighbour rows are gathered, so the only latency on
   * a row's critical path is the gathers' own; the row's x loads with its
   * own r and d after them (the same round trip), which keeps the
   * two-pack FP64 form within 64 registers: 4 CTAs of 8 warps per SM. */
  ZS_GROUP_SETUP ();
  const bool first = !PR && (flags & CHEB_FIRST), zx = flags & CHEB_ZERO_X;
  const bool wd = flags & CHEB_STORE_D, ronly = flags & CHEB_R_ONLY;
  const int64_t stride = (int64_t) gridDim.x * ngroups;
  int64_t i = (int64_t) blockIdx.x * ngroups + group;
  int64_t k0 = 0, k1 = 0;
  int mc = 0;
  T mv = T (0), mw = T (0), md = T (0);
  if (i < z.n) {
    k0 = z.rowptr[i];
    k1 = z.rowptr[i + 1];
    if (lane < k1 - k0) {
      mc = z.col[k0 + lane];
      mv = vals[k0 + lane];
      mw = vdv[k0 + lane];
      if (PR) md = dinv[mc];
    }
  }
  for (; i < z.n; i += stride) {
    const int64_t inx = i + stride;
    int64_t k0n = 0, k1n = 0;
    if (inx < z.n) {
      k0n = z.rowptr[inx];
      k1n = z.rowptr[inx + 1];
    }
    T acc[CH][W];
#pragma unroll
    for (int h = 0; h < CH; h++)
#pragma unroll
      for (int e = 0; e < W; e++) acc[h][e] = T (0);
    for (int64_t kb = k0; kb < k1; kb += G) {
      const int cnt = (int) ((k1 - kb) < G ? (k1 - kb) : G);
      if (kb != k0) {   /* rows longer than G: later chunks load inline */
        mc = 0;
        mv = mw = md = T (0);
        if (lane < cnt) {
          mc = z.col[kb + lane];
          mv = vals[kb + lane];
          mw = vdv[kb + lane];
          if (PR) md = dinv[mc];
        }
      }
      for (int t = 0; t < cnt; t++) {
        const int c = __shfl_sync (gmask, mc, t, G);
        const T av = a * __shfl_sync (gmask, mv, t, G);
        const T bw = b * __shfl_sync (gmask, mw, t, G);
        const T bpj = PR ? bp * __shfl_sync (gmask, md, t, G) : T (0);
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = lane + h * G;
          if (vi < nvec) {
            Pack<T> rj = ldp (Rold + (int64_t) c * ld + vi * W);
            Pack<T> dj = first ? pzero<T> () : ldp (Dold + (int64_t) c * ld + vi * W);
            if (PR) {
#pragma unroll
              for (int e = 0; e < W; e++) dj.v[e] = fma (bpj, dj.v[e], T (0));
            }
#pragma unroll
            for (int e = 0; e < W; e++)
              acc[h][e] = fma (bw, rj.v[e], fma (av, dj.v[e], acc[h][e]));
          }
        }
      }
    }
    /* the next row's first chunk, behind this row's gathers */
    int mcn = 0;
    T mvn = T (0), mwn = T (0), mdn = T (0);
    if (inx < z.n && lane < k1n - k0n) {
      mcn = z.col[k0n + lane];
      mvn = vals[k0n + lane];
      mwn = vdv[k0n + lane];
      if (PR) mdn = dinv[mcn];
    }
    const T bdi = b * dinv[i];
    const T bpi = PR ? bp * dinv[i] : T (0);
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        const int64_t o = i * ld + vi * W;
        Pack<T> ri = ldp (Rold + o);
        Pack<T> di = first ? pzero<T> () : ldp (Dold + o);
        Pack<T> dn, rn, x = (zx || ronly) ? pzero<T> () : ldp (X + o);
        if (PR) {
#pragma unroll
          for (int e = 0; e < W; e++) {
            di.v[e] = fma (bpi, di.v[e], T (0));   /* d_prev from r_prev */
            x.v[e] += di.v[e];         /* x_prev */
          }
        }
#pragma unroll
        for (int e = 0; e < W; e++) {
          dn.v[e] = fma (bdi, ri.v[e], a * di.v[e]);
          x.v[e] += dn.v[e];
          rn.v[e] = ri.v[e] - acc[h][e];
        }
        if (!ronly) stp (X + o, x);
        if (wd) stp (Dnew + o, dn);
        stp (Rnew + o, rn);
      }
    }
    k0 = k0n;
    k1 = k1n;
    mc = mcn;
    mv = mvn;
    mw = mwn;
    md = mdn;
  }
}

/* ---- PCG with an explicit preconditioner z = V(r) (the AMG V-cycle):
 * p_new = z + beta p_old on the fly at neighbours, q = Z p_new, (p, q) ---- */
template <typename T, int CH, bool GIVEN = false>
__global__ void __launch_bounds__ (ZS_THREADS, (CH * (16 / sizeof (T)) <= 8 ? 4 : 2))
k_pcgx_pq (ZK z, const T *__restrict__ vals, const T *__restrict__ Zb,
           const T *__restrict__ Pold, T *__restrict__ Pnew,
           T *__restrict__ Qv, int ld, int nvec, int glog, int first,
           double *partA, unsigned *counter, double *scal, int *ival, int cap)
{
  /* GIVEN: the direction p_new is already in Pnew (formed by the
   * streaming k_pcgx_pform); the product gathers p alone and Pnew is only
   * read.  Otherwise p_new = z + beta p_old is formed at every neighbour
   * row (first: p = z). */
  /* the next row's bounds and first G (column, value) pairs are loaded
   * while the current row's neighbours are gathered (software pipeline).
   * The per-column beta and each lane's running (p, q) sums live in
   * shared memory (the sums in the lane's own slots of the reduction
   * area, added to in the same row order as register sums would be), which
   * keeps the two-pack FP64 form within 64 registers: 4 CTAs per SM. */
  extern __shared__ double red[];
  ZS_GROUP_SETUP ();
  const double *beta = scal + S_BETA * cap;
  T *bsm = reinterpret_cast<T *> (red + (size_t) ngroups * ld);
  for (int c = threadIdx.x; c < ld; c += blockDim.x)
    bsm[c] = first ? T (0) : (T) beta[c];
  double *apq = red + (size_t) group * ld;
#pragma unroll
  for (int h = 0; h < CH; h++) {
    const int vi = lane + h * G;
    if (vi < nvec)
#pragma unroll
      for (int e = 0; e < W; e++) apq[vi * W + e] = 0.;
  }
  __syncthreads ();
  const int64_t stride = (int64_t) gridDim.x * ngroups;
  int64_t i = (int64_t) blockIdx.x * ngroups + group;
  int64_t k0 = 0, k1 = 0;
  int mc = 0;
  T mv = T (0);
  if (i < z.n) {
    k0 = z.rowptr[i];
    k1 = z.rowptr[i + 1];
    if (lane < k1 - k0) {
      mc = z.col[k0 + lane];
      mv = vals[k0 + lane];
    }
  }
  for (; i < z.n; i += stride) {
    const int64_t inx = i + stride;
    int64_t k0n = 0, k1n = 0;
    if (inx < z.n) {
      k0n = z.rowptr[inx];
      k1n = z.rowptr[inx + 1];
    }
    T acc[CH][W];
#pragma unroll
    for (int h = 0; h < CH; h++)
#pragma unroll
      for (int e = 0; e < W; e++) acc[h][e] = T (0);
    for (int64_t kb = k0; kb < k1; kb += G) {
      const int cnt = (int) ((k1 - kb) < G ? (k1 - kb) : G);
      if (kb != k0) {
        mc = 0;
        mv = T (0);
        if (lane < cnt) {
          mc = z.col[kb + lane];
          mv = vals[kb + lane];
        }
      }
      for (int t = 0; t < cnt; t++) {
        const int c = __shfl_sync (gmask, mc, t, G);
        const T v = __shfl_sync (gmask, mv, t, G);
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = lane + h * G;
          if (vi < nvec) {
            if constexpr (GIVEN) {
              const Pack<T> pj = ldp (Pnew + (int64_t) c * ld + vi * W);
#pragma unroll
              for (int e = 0; e < W; e++)
                acc[h][e] = fma (v, pj.v[e], acc[h][e]);
            } else {
              Pack<T> zj = ldp (Zb + (int64_t) c * ld + vi * W);
              Pack<T> pj = first ? pzero<T> () : ldp (Pold + (int64_t) c * ld + vi * W);
              const Pack<T> bt = *reinterpret_cast<const Pack<T> *> (bsm + vi * W);
#pragma unroll
              for (int e = 0; e < W; e++)
                acc[h][e] = fma (v, fma (bt.v[e], pj.v[e], zj.v[e]), acc[h][e]);
            }
          }
        }
      }
    }
    int mcn = 0;
    T mvn = T (0);
    if (inx < z.n && lane < k1n - k0n) {
      mcn = z.col[k0n + lane];
      mvn = vals[k0n + lane];
    }
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        Pack<T> pn, q;
        if constexpr (GIVEN) {
          pn = ldp (Pnew + i * ld + vi * W);
        } else {
          Pack<T> zi = ldp (Zb + i * ld + vi * W);
          Pack<T> pi = first ? pzero<T> () : ldp (Pold + i * ld + vi * W);
          const Pack<T> bt = *reinterpret_cast<const Pack<T> *> (bsm + vi * W);
#pragma unroll
          for (int e = 0; e < W; e++) pn.v[e] = fma (bt.v[e], pi.v[e], zi.v[e]);
        }
#pragma unroll
        for (int e = 0; e < W; e++) {
          q.v[e] = acc[h][e];
          apq[vi * W + e] += (double) pn.v[e] * (double) q.v[e];
        }
        if constexpr (!GIVEN) stp (Pnew + i * ld + vi * W, pn);
        stp (Qv + i * ld + vi * W, q);
      }
    }
    k0 = k0n;
    k1 = k1n;
    mc = mcn;
    mv = mvn;
  }
  __syncthreads ();
  for (int c = threadIdx.x; c < ld; c += blockDim.x) {
    double sum = 0.;
    for (int g = 0; g < ngroups; g++) sum += red[g * ld + c];
    partA[(size_t) c * gridDim.x + blockIdx.x] = sum;
  }
  const double *rz = scal + S_RZ * cap;
  double *al = scal + S_ALPHA * cap;
  int *act = ival + I_ACTIVE * cap;
  last_block_reduce (partA, ld, counter, [&] (int c, double pq) {
    if (act[c]) {
      if (pq != 0. && isfinite (pq)) al[c] = rz[c] / pq;
      else { al[c] = 0.; act[c] = 0; }
    } else {
      al[c] = 0.;
    }
  });
}

/* x += alpha p, r -= alpha q (no reductions) */
template <typename T>
__global__ void
k_pcgx_upd (int64_t n, int ld, T *__restrict__ X, T *__restrict__ R,
            const T *__restrict__ Pn,
            const T *__restrict__ Qv, const double *alpha)
{
  constexpr int W = Pack<T>::W;
  const int nvec = ld / W;
  const int64_t total = n * nvec;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / nvec;
    const int vi = (int) (e - i * nvec);
    const int64_t o = i * ld + vi * W;
    Pack<T> x = ldp (X + o), r = ldp (R + o), p = ldp (Pn + o), q = ldp (Qv + o);
#pragma unroll
    for (int k = 0; k < W; k++) {
      const T a = (T) alpha[vi * W + k];
      x.v[k] = fma (a, p.v[k], x.v[k]);
      r.v[k] = fma (-a, q.v[k], r.v[k]);
    }
    stp (X + o, x);
    stp (R + o, r);
  }
}

/* the direction, streamed: p_new = z + beta p_old; with it the previous
 * iteration's deferred x += alpha p_old (x is read by nothing inside an
 * iteration, so the update moves here from k_pcgx_upd; the same FMA, so
 * the same bits) */
template <typename T>
__global__ void
k_pcgx_pform (int64_t n, int ld, const T *__restrict__ Zb,
              const T *__restrict__ Pold, T *__restrict__ Pnew,
              T *__restrict__ X, const double *beta, const double *alpha)
{
  constexpr int W = Pack<T>::W;
  const int nvec = ld / W;
  const int64_t total = n * nvec;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / nvec;
    const int vi = (int) (e - i * nvec);
    const int64_t o = i * ld + vi * W;
    const Pack<T> z = ldp (Zb + o), p = ldp (Pold + o);
    Pack<T> x = ldp (X + o), pn;
#pragma unroll
    for (int k = 0; k < W; k++) {
      pn.v[k] = fma ((T) beta[vi * W + k], p.v[k], z.v[k]);
      x.v[k] = fma ((T) alpha[vi * W + k], p.v[k], x.v[k]);
    }
    stp (Pnew + o, pn);
    stp (X + o, x);
  }
}

/* r -= alpha q (the x half of the update is deferred to k_pcgx_pform) */
template <typename T>
__global__ void
k_pcgx_updr (int64_t n, int ld, T *__restrict__ R, const T *__restrict__ Qv,
             const double *alpha)
{
  constexpr int W = Pack<T>::W;
  const int nvec = ld / W;
  const int64_t total = n * nvec;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / nvec;
    const int vi = (int) (e - i * nvec);
    const int64_t o = i * ld + vi * W;
    Pack<T> r = ldp (R + o);
    const Pack<T> q = ldp (Qv + o);
#pragma unroll
    for (int k = 0; k < W; k++) r.v[k] = fma (-(T) alpha[vi * W + k], q.v[k], r.v[k]);
    stp (R + o, r);
  }
}

/* the last iteration's deferred x += alpha p */
template <typename T>
__global__ void
k_pcgx_xfin (int64_t n, int ld, T *__restrict__ X, const T *__restrict__ P,
             const double *alpha)
{
  constexpr int W = Pack<T>::W;
  const int nvec = ld / W;
  const int64_t total = n * nvec;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / nvec;
    const int vi = (int) (e - i * nvec);
    const int64_t o = i * ld + vi * W;
    Pack<T> x = ldp (X + o);
    const Pack<T> p = ldp (P + o);
#pragma unroll
    for (int k = 0; k < W; k++) x.v[k] = fma ((T) alpha[vi * W + k], p.v[k], x.v[k]);
    stp (X + o, x);
  }
}

/* dots (r, z), (z, z) after the preconditioner: first call sets rz, norm0
 * and the mask; later calls set beta and test convergence on ||z|| */
template <typename T, int CH>
__global__ void __launch_bounds__ (ZS_THREADS, (CH * (16 / sizeof (T)) <= 8 ? 3 : 2))
k_pcgx_dots (ZK z, const T *__restrict__ R, const T *__restrict__ Zb, int ld,
             int nvec, int glog, int w, int first, double *partA,
             double *partB, unsigned *counter, double *scal, int *ival,
             int cap, double rtol, int iter, double *hist,
             const int *fresh)
{
  extern __shared__ double red[];
  ZS_GROUP_SETUP ();
  double aRZ[CH][W], aZZ[CH][W];
#pragma unroll
  for (int h = 0; h < CH; h++)
#pragma unroll
    for (int e = 0; e < W; e++) { aRZ[h][e] = 0.; aZZ[h][e] = 0.; }
  for (int64_t i = (int64_t) blockIdx.x * ngroups + group; i < z.n;
       i += (int64_t) gridDim.x * ngroups) {
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        Pack<T> r = ldp (R + i * ld + vi * W), zz = ldp (Zb + i * ld + vi * W);
#pragma unroll
        for (int e = 0; e < W; e++) {
          aRZ[h][e] += (double) r.v[e] * (double) zz.v[e];
          aZZ[h][e] += (double) zz.v[e] * (double) zz.v[e];
        }
      }
    }
  }
  block_colsum_store<T, CH> (aRZ, lane, group, G, nvec, ld, red, partA);
  block_colsum_store<T, CH> (aZZ, lane, group, G, nvec, ld, red, partB);
  double *rz = scal + S_RZ * cap, *be = scal + S_BETA * cap;
  double *al_g = scal + S_ALPHA * cap, *n0 = scal + S_NORM0 * cap;
  int *act = ival + I_ACTIVE * cap, *its = ival + I_ITS * cap;
  bool last = last_block_reduce2 (partA, partB, ld, counter,
      [&] (int c, double srz, double szz) {
        if (first || (fresh != nullptr && fresh[c])) {
          rz[c] = srz;
          n0[c] = sqrt (szz);
          act[c] = (c < w && szz > 0.) ? 1 : 0;
          al_g[c] = 0.;
          be[c] = 0.;
          its[c] = 0;
          return;
        }
        if (!act[c]) { be[c] = 0.; return; }
        const double b = (rz[c] != 0.) ? srz / rz[c] : 0.;
        if (hist != nullptr && c == 0 && iter < 10000) {
          hist[2 * iter] = al_g[0];
          hist[2 * iter + 1] = b;
        }
        rz[c] = srz;
        be[c] = b;
        /* a converged column keeps its alpha: its x update may still be
         * pending (k_pcgx_pform or k_pcgx_xfin applies it), and the next
         * product zeroes alpha for inactive columns */
        if (sqrt (szz) <= rtol * n0[c] || srz == 0.) {
          act[c] = 0;
          be[c] = 0.;
          its[c] = iter + 1;
        }
      });
  if (last) {
    __syncthreads ();
    if (threadIdx.x == 0) {
      int cnt = 0;
      for (int c = 0; c < ld; c++) cnt += act[c];
      ival[I_NSLOT * cap] = cnt;
    }
  }
}

/* Chebyshev with an explicit preconditioner: d_new = a d + b z on the fly
 * at neighbours, x += d_new, r_new = r - Z d_new */
template <typename T, int CH>
__global__ void __launch_bounds__ (ZS_THREADS, (CH * (16 / sizeof (T)) <= 8 ? 3 : 2))
k_chebx (ZK z, const T *__restrict__ vals, const T *__restrict__ Zb,
         T *__restrict__ X,
         const T *__restrict__ Rold, T *__restrict__ Rnew,
         const T *__restrict__ Dold, T *__restrict__ Dnew, int ld, int nvec,
         int glog, T a, T b, int first)
{
  ZS_GROUP_SETUP ();
  for (int64_t i = (int64_t) blockIdx.x * ngroups + group; i < z.n;
       i += (int64_t) gridDim.x * ngroups) {
    T acc[CH][W];
#pragma unroll
    for (int h = 0; h < CH; h++)
#pragma unroll
      for (int e = 0; e < W; e++) acc[h][e] = T (0);
    const int64_t k0 = z.rowptr[i], k1 = z.rowptr[i + 1];
    for (int64_t kb = k0; kb < k1; kb += G) {
      const int cnt = (int) ((k1 - kb) < G ? (k1 - kb) : G);
      int mc = 0;
      T mv = T (0);
      if (lane < cnt) {
        mc = z.col[kb + lane];
        mv = vals[kb + lane];
      }
      for (int t = 0; t < cnt; t++) {
        const int c = __shfl_sync (gmask, mc, t, G);
        const T v = __shfl_sync (gmask, mv, t, G);
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = lane + h * G;
          if (vi < nvec) {
            Pack<T> zj = ldp (Zb + (int64_t) c * ld + vi * W);
            Pack<T> dj = first ? pzero<T> () : ldp (Dold + (int64_t) c * ld + vi * W);
#pragma unroll
            for (int e = 0; e < W; e++)
              acc[h][e] = fma (v, fma (b, zj.v[e], a * dj.v[e]), acc[h][e]);
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        const int64_t o = i * ld + vi * W;
        Pack<T> ri = ldp (Rold + o), x = ldp (X + o), zi = ldp (Zb + o);
        Pack<T> di = first ? pzero<T> () : ldp (Dold + o);
        Pack<T> dn, rn;
#pragma unroll
        for (int e = 0; e < W; e++) {
          dn.v[e] = fma (b, zi.v[e], a * di.v[e]);
          x.v[e] += dn.v[e];
          rn.v[e] = ri.v[e] - acc[h][e];
        }
        stp (X + o, x);
        stp (Dnew + o, dn);
        stp (Rnew + o, rn);
      }
    }
  }
}

/* ---- FP64 residual, R = S B - Z X (pads zero), per-column ||D^{-1} R|| and
 * ||D^{-1} S B|| (tests) ------------------------------------------------- */
template <typename TO, int CH>
__global__ void __launch_bounds__ (ZS_THREADS)
k_zresid (ZK z, const double *__restrict__ vals,
          const double *__restrict__ dinv, const double *__restrict__ Bm,
          int ldb, const double *__restrict__ rs_in,
          const double *__restrict__ X, int ldx, TO *Rout, int ldr, int nvec,
          int glog, int w, double *partA, double *partB, unsigned *counter,
          double *out_r, double *out_b)
{
  extern __shared__ double red[];
  using T = double;
  ZS_GROUP_SETUP ();
  double aR[CH][W], aB[CH][W];
#pragma unroll
  for (int h = 0; h < CH; h++)
#pragma unroll
    for (int e = 0; e < W; e++) { aR[h][e] = 0.; aB[h][e] = 0.; }
  const int ld = nvec * W;
  for (int64_t i = (int64_t) blockIdx.x * ngroups + group; i < z.n;
       i += (int64_t) gridDim.x * ngroups) {
    double acc[CH][W];
#pragma unroll
    for (int h = 0; h < CH; h++)
#pragma unroll
      for (int e = 0; e < W; e++) acc[h][e] = 0.;
    for (int64_t k = z.rowptr[i]; k < z.rowptr[i + 1]; k++) {
      const int c = z.col[k];
      const double v = vals[k];
#pragma unroll
      for (int h = 0; h < CH; h++) {
        const int vi = lane + h * G;
        if (vi < nvec) {
          Pack<double> xj = ldp (X + (int64_t) c * ldx + vi * W);
#pragma unroll
          for (int e = 0; e < W; e++) acc[h][e] = fma (v, xj.v[e], acc[h][e]);
        }
      }
    }
    const double sc = rs_in ? rs_in[i] : 1.0, di = dinv[i];
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
#pragma unroll
        for (int e = 0; e < W; e++) {
          const int c = vi * W + e;
          const double bv = (c < w) ? sc * Bm[i * ldb + c] : 0.;
          const double r = (c < w) ? bv - acc[h][e] : 0.;
          aR[h][e] += (di * r) * (di * r);
          aB[h][e] += (di * bv) * (di * bv);
          if (Rout) Rout[i * ldr + c] = (TO) r;
        }
      }
    }
  }
  if (out_r == nullptr) return;
  block_colsum_store<double, CH> (aR, lane, group, G, nvec, ld, red, partA);
  block_colsum_store<double, CH> (aB, lane, group, G, nvec, ld, red, partB);
  last_block_reduce2 (partA, partB, ld, counter,
                      [&] (int c, double sr, double sb) {
                        out_r[c] = sqrt (sr);
                        if (out_b) out_b[c] = sqrt (sb);
                      });
}

/* ---- host side ------------------------------------------------------------ */

/* opt a kernel into > 48 KB of dynamic shared memory, once per kernel */
static void
smem_prep (const void *fn, int bytes)
{
  static std::mutex mu;
  static std::unordered_map<const void *, int> done;
  if (bytes <= 48 * 1024) return;
  std::lock_guard<std::mutex> lk (mu);
  auto it = done.find (fn);
  if (it != done.end () && it->second >= bytes) return;
  cudaFuncSetAttribute (fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        bytes);
  done[fn] = bytes;
}

template <typename K>
static void
set_smem_attr (K kern, int bytes)
{
  smem_prep ((const void *) kern, bytes);
}

static int
zs_smem_bytes (int glog, int ld)
{
  return (ZS_THREADS >> glog) * ld * (int) sizeof (double);
}

/* k_pcgx_pq: the reduction area plus the per-column beta */
static int
zs_pq_smem_bytes (int glog, int ld)
{
  return zs_smem_bytes (glog, ld) + ld * (int) sizeof (double);
}

int
ZWork::alloc (int64_t n_, int cap_, int is32_)
{
  cap_ = round_ld (cap_);
  if (n_ == n && cap_ <= cap && is32_ == is32 && X.p) return 0;
  n = n_;
  cap = cap_;
  is32 = is32_;
  const size_t es = is32 ? 4 : 8;
  const size_t blk = (size_t) n * cap * es;
  LGH_TRY (X.alloc (blk));
  LGH_TRY (R.alloc (blk));
  LGH_TRY (P0.alloc (blk));
  LGH_TRY (P1.alloc (blk));
  LGH_TRY (Q.alloc (blk));
  LGH_TRY (Zb.alloc (blk));
  nblocks = num_sms () * 8;
  LGH_TRY (partA.alloc ((size_t) cap * nblocks));
  LGH_TRY (partB.alloc ((size_t) cap * nblocks));
  LGH_TRY (scal.alloc ((size_t) cap * S_NSLOT));
  LGH_TRY (ival.alloc ((size_t) cap * I_NSLOT + 8));
  LGH_TRY (counters.alloc (8));
  LGH_TRY (hist.alloc (2 * 10000 + 16));
  LGH_CUDA (cudaMemset (counters.p, 0, 8 * sizeof (unsigned)));
  LGH_CUDA (cudaMemset (ival.p, 0, ((size_t) cap * I_NSLOT + 8) * sizeof (int)));
  return 0;
}

template <typename T>
static const T *
zvals (const Csr &Z)
{
  if constexpr (std::is_same<T, double>::value) return Z.vals;
  else return Z.vals32;
}

template <typename T>
static const T *
zdinv (const Csr &Z)
{
  if constexpr (std::is_same<T, double>::value) return Z.dinv;
  else return Z.dinv32;
}

template <typename T>
static const T *
zvd (const Csr &Z)
{
  if constexpr (std::is_same<T, double>::value) return Z.vd;
  else return Z.vd32;
}

#define ZS_DISPATCH(CHV, ...)                                                \
  switch (CHV) {                                                             \
  case 1: { constexpr int CH_ = 1; __VA_ARGS__; } break;                     \
  case 2: { constexpr int CH_ = 2; __VA_ARGS__; } break;                     \
  case 3: { constexpr int CH_ = 3; __VA_ARGS__; } break;                     \
  case 4: { constexpr int CH_ = 4; __VA_ARGS__; } break;                     \
  case 5: { constexpr int CH_ = 5; __VA_ARGS__; } break;                     \
  case 6: { constexpr int CH_ = 6; __VA_ARGS__; } break;                     \
  case 7: { constexpr int CH_ = 7; __VA_ARGS__; } break;                     \
  case 8: { constexpr int CH_ = 8; __VA_ARGS__; } break;                     \
  default:                                                                   \
    return set_error (LGH_ERR_SUP, "zsolve: chunking %d unsupported", CHV);  \
  }

/* flat conversion of a row-major block (same leading dimension on both
 * sides), four elements per thread */
template <typename TI, typename TO>
__global__ void
k_cvt_flat (int64_t count, const TI *__restrict__ X, TO *__restrict__ Y)
{
  const int64_t q = count / 4;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < q;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t o = e * 4;
#pragma unroll
    for (int k = 0; k < 4; k++) Y[o + k] = (TO) X[o + k];
  }
  for (int64_t o = q * 4 + (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
       o < count; o += (int64_t) gridDim.x * blockDim.x)
    Y[o] = (TO) X[o];
}

template <typename TI, typename TO>
int
cvt_flat (int64_t count, const TI *X, TO *Y, cudaStream_t s)
{
  const int grid = (int) std::max<int64_t> (1, std::min<int64_t> (
      (int64_t) num_sms () * 8, (count / 4 + 255) / 256));
  k_cvt_flat<TI, TO><<<grid, 256, 0, s>>> (count, X, Y);
  LGH_LAUNCH_CHECK ();
  return 0;
}

template int cvt_flat<double, float> (int64_t, const double *, float *,
                                      cudaStream_t);
template int cvt_flat<float, double> (int64_t, const float *, double *,
                                      cudaStream_t);

template <typename T>
int
zsolve_block (const Csr &Z, const ZsolveCfg &cfg, Hierarchy *mg, ZWork &ws,
              int64_t n, int w, const T *Xin, int ldx,
              const double *rs_in, T *Y, int ldy, const double *rs_out,
              ZsolveStats *st, int record_hist, cudaStream_t s)
{
  constexpr int W = Pack<T>::W;
  (void) mg;
  if (w <= 0 || n == 0) return 0;
  LGH_CHECK (cfg.mode != 3 || mg != nullptr, LGH_ERR_SUP,
             "zsolve: mode 3 needs the multigrid preconditioner");
  LGH_CHECK (Z.dinv != nullptr, LGH_ERR_ARG_WRONGSTATE, "zsolve: Z has no diagonal");
  const double t0 = wall ();
  int tile = ws.cap;
  if (cfg.mode >= 2 && cfg.tile > 0) tile = std::min (tile, round_ld (cfg.tile));
  tile = std::max (4, tile & ~3);
  /* FP32 tiles stop at 4 chunks per lane (their FP64 dot accumulators
   * would spill beyond that) */
  const int maxcols = 32 * (sizeof (T) == 4 ? 4 : ZS_MAXCH) * W;
  tile = std::min (tile, maxcols);
  const T *vals = zvals<T> (Z);
  const T *dinv = zdinv<T> (Z);
  ZK zk{ Z.n, Z.rowptr, Z.colidx };
  /* optional per-kernel event timing (lgh_kernel_timing) */
  const bool timing = ktime_on ();
  static thread_local EventRing ring;
  std::vector<int> tids;
  std::vector<double> tbytes;
  const double zbytes = (double) Z.nnz * (sizeof (T) + 4) + 8. * (Z.n + 1)
                        + (double) Z.n * sizeof (T);
  T *bX = (T *) ws.X.p, *bR = (T *) ws.R.p, *bP0 = (T *) ws.P0.p,
    *bP1 = (T *) ws.P1.p, *bQ = (T *) ws.Q.p;
  std::vector<int> its_h;

  for (int c0 = 0; c0 < w; c0 += tile) {
    const int wt = std::min (tile, w - c0);
    const int ldt = round_ld (wt);
    const int nvec = ldt / W;
    int glog, ch;
    row_group_shape (nvec, glog, ch, Z.max_row_nnz);
    const int grid = std::min (row_grid (n, glog), ws.nblocks);
    const int smem = zs_smem_bytes (glog, ldt);
    const int cap = ws.cap;
    int *nact = ws.ival.p + I_NSLOT * cap;

    ZS_DISPATCH (ch, {
      auto kf = k_pcg_init<T, CH_>;
      set_smem_attr (kf, smem);
      kf<<<fit_grid (kf, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, dinv, Xin + c0, ldx, rs_in, bX,
                                         bR, bP0, ldt, nvec, glog, wt,
                                         ws.partA.p, ws.partB.p,
                                         ws.counters.p, ws.scal.p, ws.ival.p,
                                         cap);
    });
    LGH_LAUNCH_CHECK ();

    int iters = 0;
    T *bZ = (T *) ws.Zb.p;
    if (cfg.mode <= 1 && mg != nullptr) {
      /* PCG with the V-cycle: z = V(r) each iteration (the reference's
       * per-column CG + PCGAMG, zsolve_impl.h:674-683, 808-818) */
      const int egrid = std::max (1, std::min (num_sms () * 8,
                                  (int) ((n * (ldt / W) + 255) / 256)));
      static thread_local KTrace ktr;
      KTrace *tr = timing ? &ktr : nullptr;
      const double bw = (double) n * wt * sizeof (T);
      /* z = V(r): in T, or (cfg.pc32, FP64 iterates) an FP32 V-cycle
       * between two conversions: the Krylov vectors and so the attainable
       * accuracy stay FP64, the V-cycle's traffic is halved */
      const bool pc32 = cfg.pc32 && std::is_same<T, double>::value;
      float *R32 = nullptr, *Z32 = nullptr;
      if (pc32) {
        LGH_TRY (ws.R32.alloc ((size_t) n * ws.cap * sizeof (float)));
        LGH_TRY (ws.Z32.alloc ((size_t) n * ws.cap * sizeof (float)));
        R32 = (float *) ws.R32.p;
        Z32 = (float *) ws.Z32.p;
      }
      auto precond = [&] () -> int {
        if (!pc32) return mg_vcycle<T> (mg, bR, bZ, ldt, wt, s, tr);
        const int64_t cnt = n * (int64_t) ldt;
        LGH_TRY ((cvt_flat<T, float> (cnt, bR, R32, s)));
        LGH_TRY (mg_vcycle<float> (mg, R32, Z32, ldt, wt, s, nullptr));
        return cvt_flat<float, T> (cnt, Z32, bZ, s);
      };
      LGH_TRY (precond ());
      ZS_DISPATCH (ch, {
        auto kd = k_pcgx_dots<T, CH_>;
        set_smem_attr (kd, smem);
        kd<<<fit_grid (kd, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, bR, bZ, ldt, nvec, glog, wt, 1,
                                           ws.partA.p, ws.partB.p,
                                           ws.counters.p + 1, ws.scal.p,
                                           ws.ival.p, cap, cfg.rtol, 0, nullptr, nullptr);
      });
      LGH_LAUNCH_CHECK ();
      T *Pold = bP0, *Pnew = bP1;
      int h_nact = 1;
      const double *alpha = ws.scal.p + S_ALPHA * cap;
      const double *betap = ws.scal.p + S_BETA * cap;
      for (int it = 0; it < cfg.maxit; it++) {
        /* iteration 0: p = z inside the product; later iterations: the
         * direction p = z + beta p_old by a streaming pass, which also
         * applies the previous iteration's x += alpha p_old, then the
         * product gathers p alone */
        if (it > 0) {
          if (tr) LGH_TRY (tr->begin (K_PCGX_PFORM, 5. * bw, s));
          k_pcgx_pform<T><<<egrid, 256, 0, s>>> (n, ldt, bZ, Pold, Pnew, bX,
                                                betap, alpha);
          LGH_LAUNCH_CHECK ();
          if (tr) LGH_TRY (tr->end (s));
        }
        if (tr) LGH_TRY (tr->begin (K_PCGX_PQ, zbytes + (it == 0 ? 3. : 2.) * bw, s));
        ZS_DISPATCH (ch, {
          const int psm = zs_pq_smem_bytes (glog, ldt);
          if (it == 0) {
            auto k1 = k_pcgx_pq<T, CH_, false>;
            set_smem_attr (k1, psm);
            k1<<<fit_grid (k1, grid, ZS_THREADS, psm), ZS_THREADS, psm, s>>> (
                zk, vals, bZ, Pold, Pnew, bQ, ldt, nvec, glog, 1, ws.partA.p,
                ws.counters.p, ws.scal.p, ws.ival.p, cap);
          } else {
            auto k1 = k_pcgx_pq<T, CH_, true>;
            set_smem_attr (k1, psm);
            k1<<<fit_grid (k1, grid, ZS_THREADS, psm), ZS_THREADS, psm, s>>> (
                zk, vals, bZ, Pold, Pnew, bQ, ldt, nvec, glog, 0, ws.partA.p,
                ws.counters.p, ws.scal.p, ws.ival.p, cap);
          }
        });
        LGH_LAUNCH_CHECK ();
        if (tr) LGH_TRY (tr->end (s));
        if (tr) LGH_TRY (tr->begin (K_PCGX_UPD, 3. * bw, s));
        k_pcgx_updr<T><<<egrid, 256, 0, s>>> (n, ldt, bR, bQ, alpha);
        LGH_LAUNCH_CHECK ();
        if (tr) LGH_TRY (tr->end (s));
        LGH_TRY (precond ());
        if (tr) LGH_TRY (tr->begin (K_PCGX_DOTS, 2. * bw, s));
        ZS_DISPATCH (ch, {
          auto kd = k_pcgx_dots<T, CH_>;
          kd<<<fit_grid (kd, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, bR, bZ, ldt, nvec, glog, wt, 0,
                                             ws.partA.p, ws.partB.p,
                                             ws.counters.p + 1, ws.scal.p,
                                             ws.ival.p, cap, cfg.rtol, it,
                                             record_hist ? ws.hist.p : nullptr,
                                             nullptr);
        });
        LGH_LAUNCH_CHECK ();
        if (tr) LGH_TRY (tr->end (s));
        std::swap (Pold, Pnew);
        iters = it + 1;
        if (iters % 2 == 0 || iters == cfg.maxit || iters <= 2) {
          LGH_CUDA (cudaMemcpyAsync (&h_nact, nact, sizeof (int),
                                     cudaMemcpyDeviceToHost, s));
          LGH_CUDA (cudaStreamSynchronize (s));
          if (tr) LGH_TRY (tr->drain ());
          if (h_nact == 0) break;
        }
      }
      /* the last iteration's deferred x += alpha p (its direction is in
       * Pold after the swap) */
      k_pcgx_xfin<T><<<egrid, 256, 0, s>>> (n, ldt, bX, Pold, alpha);
      LGH_LAUNCH_CHECK ();
      if (tr && !tr->ids.empty ()) {
        LGH_CUDA (cudaStreamSynchronize (s));
        LGH_TRY (tr->drain ());
      }
      if (st) {
        its_h.resize (ldt);
        std::vector<int> act_h (ldt);
        LGH_CUDA (cudaMemcpyAsync (its_h.data (), ws.ival.p + I_ITS * cap,
                                   ldt * sizeof (int), cudaMemcpyDeviceToHost, s));
        LGH_CUDA (cudaMemcpyAsync (act_h.data (), ws.ival.p + I_ACTIVE * cap,
                                   ldt * sizeof (int), cudaMemcpyDeviceToHost, s));
        LGH_CUDA (cudaStreamSynchronize (s));
        for (int c = 0; c < wt; c++) st->col_iters += act_h[c] ? iters : its_h[c];
        if (h_nact > 0) st->last_maxit_hit = 1;
        st->cols += wt;
      }
    } else if (cfg.mode >= 2 && mg != nullptr) {
      /* Chebyshev around the V-cycle (modes 2/3: zsolve_impl.h:108-141
       * with the AMG / harvested-hierarchy preconditioner) */
      const double theta = 0.5 * (cfg.lmax + cfg.lmin);
      const double delta = 0.5 * (cfg.lmax - cfg.lmin);
      const double sigma1 = theta / delta;
      double rho_old = 1.0 / sigma1;
      T *Ro = bR, *Rn = bQ, *Do = bP0, *Dn = bP1;
      for (int k = 1; k <= cfg.nit; k++) {
        double a, b;
        if (k == 1) { a = 0.; b = 1.0 / theta; }
        else {
          const double rho = 1.0 / (2.0 * sigma1 - rho_old);
          a = rho * rho_old;
          b = 2.0 * rho / delta;
          rho_old = rho;
        }
        static thread_local KTrace ktc;
        KTrace *tc = (timing && k % 4 == 0) ? &ktc : nullptr;
        LGH_TRY (mg_vcycle<T> (mg, Ro, bZ, ldt, wt, s, tc));
        if (tc) LGH_TRY (tc->begin (K_CHEBX, zbytes + 7. * (double) n * wt * sizeof (T), s));
        ZS_DISPATCH (ch, {
          k_chebx<T, CH_><<<fit_grid (k_chebx<T, CH_>, grid, ZS_THREADS, 0),
                                           ZS_THREADS, 0, s>>> (zk, vals, bZ, bX, Ro, Rn,
                                                       Do, Dn, ldt, nvec, glog,
                                                       (T) a, (T) b,
                                                      (k == 1 ? CHEB_FIRST : 0)
                                                      | CHEB_STORE_D);
        });
        LGH_LAUNCH_CHECK ();
        if (tc) {
          LGH_TRY (tc->end (s));
          LGH_CUDA (cudaStreamSynchronize (s));
          LGH_TRY (tc->drain ());
        }
        std::swap (Ro, Rn);
        std::swap (Do, Dn);
      }
      iters = cfg.nit;
      if (st) { st->col_iters += (long) iters * wt; st->cols += wt; }
    } else if (cfg.mode <= 1) {
      T *Pold = bP0, *Pnew = bP1;
      int h_nact = 1;
      const double bw = (double) n * wt * sizeof (T);
      for (int it = 0; it < cfg.maxit; it++) {
        if (timing) {
          LGH_TRY (ring.record (s));
          tids.push_back (K_PCG_PQ);
          tbytes.push_back (zbytes + (it == 0 ? 3. : 4.) * bw);
        }
        ZS_DISPATCH (ch, {
          auto k1 = k_pcg_pq<T, CH_>;
          set_smem_attr (k1, smem);
          k1<<<fit_grid (k1, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, vals, dinv, bR, Pold, Pnew,
                                             bQ, ldt, nvec, glog, it == 0,
                                             ws.partA.p, ws.counters.p,
                                             ws.scal.p, ws.ival.p, cap);
          if (timing) {
            LGH_TRY (ring.record (s));
            tids.push_back (K_PCG_UPD);
            tbytes.push_back (6. * bw + (double) n * sizeof (T));
          }
          auto k2 = k_pcg_upd<T, CH_>;
          set_smem_attr (k2, smem);
          k2<<<fit_grid (k2, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, dinv, bX, bR, Pnew, bQ, ldt,
                                             nvec, glog, ws.partA.p,
                                             ws.partB.p, ws.counters.p + 1,
                                             ws.scal.p, ws.ival.p, cap,
                                             cfg.rtol, it,
                                             record_hist ? ws.hist.p : nullptr);
        });
        LGH_LAUNCH_CHECK ();
        if (timing) {
          LGH_TRY (ring.record (s));
          tids.push_back (-1);
          tbytes.push_back (0.);
        }
        std::swap (Pold, Pnew);
        iters = it + 1;
        if (iters % cfg.check_every == 0 || iters == cfg.maxit || iters <= 2) {
          LGH_CUDA (cudaMemcpyAsync (&h_nact, nact, sizeof (int),
                                     cudaMemcpyDeviceToHost, s));
          LGH_CUDA (cudaStreamSynchronize (s));
          if (timing) {
            LGH_TRY (ring.drain (tids, tbytes));
            tids.clear ();
            tbytes.clear ();
          }
          if (h_nact == 0) break;
        }
      }
      if (timing && !tids.empty ()) {
        LGH_CUDA (cudaStreamSynchronize (s));
        LGH_TRY (ring.drain (tids, tbytes));
        tids.clear ();
        tbytes.clear ();
      }
      if (st) {
        its_h.resize (ldt);
        LGH_CUDA (cudaMemcpyAsync (its_h.data (), ws.ival.p + I_ITS * cap,
                                   ldt * sizeof (int), cudaMemcpyDeviceToHost, s));
        std::vector<int> act_h (ldt);
        LGH_CUDA (cudaMemcpyAsync (act_h.data (), ws.ival.p + I_ACTIVE * cap,
                                   ldt * sizeof (int), cudaMemcpyDeviceToHost, s));
        LGH_CUDA (cudaStreamSynchronize (s));
        for (int c = 0; c < wt; c++) st->col_iters += act_h[c] ? iters : its_h[c];
        if (h_nact > 0) st->last_maxit_hit = 1;
        st->cols += wt;
      }
    } else {
      /* Chebyshev, fixed count (zsolve_impl.h:113-139) */
      const double theta = 0.5 * (cfg.lmax + cfg.lmin);
      const double delta = 0.5 * (cfg.lmax - cfg.lmin);
      const double sigma1 = theta / delta;
      double rho_old = 1.0 / sigma1;
      T *Ro = bR, *Rn = bQ, *Do = bP0, *Dn = bP1;
      for (int k = 1; k <= cfg.nit; k++) {
        double a, b;
        if (k == 1) { a = 0.; b = 1.0 / theta; }
        else {
          const double rho = 1.0 / (2.0 * sigma1 - rho_old);
          a = rho * rho_old;
          b = 2.0 * rho / delta;
          rho_old = rho;
        }
        const bool tk = timing && (k % 8 == 0);
        if (tk) {
          LGH_TRY (ring.record (s));
          tids.push_back (K_CHEB);
          tbytes.push_back (zbytes + 6. * (double) n * wt * sizeof (T));
        }
        LGH_TRY (launch_cheb_step<T> (Z, bX, Ro, Rn, Do, Dn, ldt, a, b,
                                      (k == 1 ? CHEB_FIRST : 0) | CHEB_STORE_D, s));
        if (tk) {
          LGH_TRY (ring.record (s));
          tids.push_back (-1);
          tbytes.push_back (0.);
        }
        std::swap (Ro, Rn);
        std::swap (Do, Dn);
      }
      iters = cfg.nit;
      if (timing && !tids.empty ()) {
        LGH_CUDA (cudaStreamSynchronize (s));
        LGH_TRY (ring.drain (tids, tbytes));
        tids.clear ();
        tbytes.clear ();
      }
      if (st) { st->col_iters += (long) iters * wt; st->cols += wt; }
    }
    if (st) st->block_iters += iters;
    LGH_TRY (launch_rowscale<T> (n, wt, rs_out, bX, ldt, Y + c0, ldy, s));
  }
  if (st) {
    LGH_CUDA (cudaStreamSynchronize (s));
    st->calls++;
    st->seconds += wall () - t0;
  }
  return 0;
}

template int zsolve_block<double> (const Csr &, const ZsolveCfg &, Hierarchy *,
                                   ZWork &, int64_t, int, const double *, int,
                                   const double *, double *, int,
                                   const double *, ZsolveStats *, int,
                                   cudaStream_t);
template int zsolve_block<float> (const Csr &, const ZsolveCfg &, Hierarchy *,
                                  ZWork &, int64_t, int, const float *, int,
                                  const double *, float *, int, const double *,
                                  ZsolveStats *, int, cudaStream_t);

/* ---- one tick of the request loop's slot block (server.cu) ------------- */

template <typename T>
int
server_tick_pq (const Csr &Z, const T *Zb, const T *Pold, T *Pnew, T *Q, int ld,
                ZWork &ws, cudaStream_t s)
{
  constexpr int W = Pack<T>::W;
  const int nvec = ld / W;
  int glog, ch;
  row_group_shape (nvec, glog, ch, Z.max_row_nnz);
  const int grid = std::min (row_grid (Z.n, glog), ws.nblocks);
  const int smem = zs_pq_smem_bytes (glog, ld);
  ZK zk{ Z.n, Z.rowptr, Z.colidx };
  ZS_DISPATCH (ch, {
    auto k1 = k_pcgx_pq<T, CH_>;
    set_smem_attr (k1, smem);
    k1<<<fit_grid (k1, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, zvals<T> (Z), Zb, Pold, Pnew, Q, ld,
                                       nvec, glog, 0, ws.partA.p,
                                       ws.counters.p, ws.scal.p, ws.ival.p,
                                       ws.cap);
  });
  LGH_LAUNCH_CHECK ();
  return 0;
}

template <typename T>
int
server_tick_upd (int64_t n, int ld, T *X, T *R, const T *Pn, const T *Q,
                 ZWork &ws, cudaStream_t s)
{
  constexpr int W = Pack<T>::W;
  const int egrid = std::max (1, std::min (num_sms () * 8,
                              (int) ((n * (ld / W) + 255) / 256)));
  k_pcgx_upd<T><<<egrid, 256, 0, s>>> (n, ld, X, R, Pn, Q,
                                       ws.scal.p + S_ALPHA * ws.cap);
  LGH_LAUNCH_CHECK ();
  return 0;
}

template <typename T>
int
server_tick_dots (const Csr &Z, const T *R, const T *Zb, int ld, int w,
                  const int *fresh, double rtol, ZWork &ws, cudaStream_t s)
{
  constexpr int W = Pack<T>::W;
  const int nvec = ld / W;
  int glog, ch;
  row_group_shape (nvec, glog, ch, Z.max_row_nnz);
  const int grid = std::min (row_grid (Z.n, glog), ws.nblocks);
  const int smem = zs_smem_bytes (glog, ld);
  ZK zk{ Z.n, Z.rowptr, Z.colidx };
  ZS_DISPATCH (ch, {
    auto kd = k_pcgx_dots<T, CH_>;
    set_smem_attr (kd, smem);
    kd<<<fit_grid (kd, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, R, Zb, ld, nvec, glog, w, 0,
                                       ws.partA.p, ws.partB.p,
                                       ws.counters.p + 1, ws.scal.p, ws.ival.p,
                                       ws.cap, rtol, 0, nullptr, fresh);
  });
  LGH_LAUNCH_CHECK ();
  return 0;
}

template int server_tick_pq<double> (const Csr &, const double *, const double *,
                                     double *, double *, int, ZWork &,
                                     cudaStream_t);
template int server_tick_upd<double> (int64_t, int, double *, double *,
                                      const double *, const double *, ZWork &,
                                      cudaStream_t);
template int server_tick_dots<double> (const Csr &, const double *,
                                       const double *, int, int, const int *,
                                       double, ZWork &, cudaStream_t);

/* L2 bytes the smoother's neighbour reuse may span: a row's r and d rows
 * are gathered again by the rows up to the bandwidth away, so the band of
 * 2 bandwidth rows of both blocks must stay in L2 (126 MB, shared with the
 * streaming writes).  A wider band is swept in column slices.
 * LGH_CHEB_L2MB overrides the budget (0: never slice). */
static double
cheb_l2_budget ()
{
  const char *e = getenv ("LGH_CHEB_L2MB");
  return (e ? atof (e) : 40.0) * 1048576.0;
}

/* one Chebyshev-Jacobi step on a CSR operator (the multigrid smoother and
 * the fixed-count Chebyshev mode) */
template <typename T>
int
launch_cheb_step (const Csr &A, T *X, const T *Ro, T *Rn, const T *Do, T *Dn,
                  int ld, double a, double b, int flags, cudaStream_t s,
                  double bp)
{
  constexpr int W = Pack<T>::W;
  const int nvec_all = ld / W;
  ZK zk{ A.n, A.rowptr, A.colidx };
  const T *vals = zvals<T> (A);
  const T *dinv = zdinv<T> (A);
  /* column slices of whole packs so that each slice's reuse band fits */
  const double band = 2. * 2. * (double) A.bandwidth * ld * sizeof (T);
  const double budget = cheb_l2_budget ();
  int slices = 1;
  if (budget > 0. && band > budget)
    slices = std::min (nvec_all, (int) std::ceil (band / budget));
  for (int sl = 0; sl < slices; sl++) {
    const int v0 = (int) ((int64_t) nvec_all * sl / slices);
    const int v1 = (int) ((int64_t) nvec_all * (sl + 1) / slices);
    const int nvec = v1 - v0;
    if (nvec <= 0) continue;
    const int c0 = v0 * W;
    int glog, ch;
    row_group_shape (nvec, glog, ch, A.max_row_nnz);
    const int grid = std::min (row_grid (A.n, glog), num_sms () * 8);
    ZS_DISPATCH (ch, {
      if (flags & CHEB_PREV_R) {
        auto k = k_cheb<T, CH_, true>;
        k<<<fit_grid (k, grid, ZS_THREADS, 0), ZS_THREADS, 0, s>>> (
            zk, vals, zvd<T> (A), dinv, X + c0, Ro + c0, Rn + c0, Do + c0,
            Dn ? Dn + c0 : nullptr, ld, nvec, glog, (T) a, (T) b, flags,
            (T) bp);
      } else {
        auto k = k_cheb<T, CH_, false>;
        k<<<fit_grid (k, grid, ZS_THREADS, 0), ZS_THREADS, 0, s>>> (
            zk, vals, zvd<T> (A), dinv, X + c0, Ro + c0, Rn + c0,
            Do ? Do + c0 : nullptr, Dn ? Dn + c0 : nullptr, ld, nvec, glog,
            (T) a, (T) b, flags, T (0));
      }
    });
    LGH_LAUNCH_CHECK ();
  }
  return 0;
}

/* the last Chebyshev step of a smoothing sequence whose residual is not
 * needed afterwards: x += a d + b D^{-1} r, elementwise (no Z product) */
template <typename T>
__global__ void
k_cheb_tail (int64_t n, int ld, const T *__restrict__ dinv, T *__restrict__ X,
             const T *__restrict__ R, const T *__restrict__ D, T a, T b,
             int first, int prevr, T bp)
{
  /* prevr: D holds the residual of a first step (coefficient bp) that
   * stored only its residual; its d and x are formed here with that
   * step's roundings (d_prev = (bp dinv_i) r_prev, x_prev = x + d_prev) */
  constexpr int W = Pack<T>::W;
  const int nvec = ld / W;
  const int64_t total = n * nvec;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / nvec;
    const int64_t o = i * ld + (e - i * nvec) * W;
    const T bdi = b * dinv[i];
    Pack<T> x = ldp (X + o), r = ldp (R + o);
    Pack<T> d = first ? pzero<T> () : ldp (D + o);
    if (prevr) {
      const T bpi = bp * dinv[i];
#pragma unroll
      for (int k = 0; k < W; k++) {
        d.v[k] = fma (bpi, d.v[k], T (0));
        x.v[k] += d.v[k];
      }
    }
#pragma unroll
    for (int k = 0; k < W; k++) x.v[k] += fma (bdi, r.v[k], a * d.v[k]);
    stp (X + o, x);
  }
}

template <typename T>
int
launch_cheb_tail (const Csr &A, T *X, const T *R, const T *D, int ld, double a,
                  double b, int first, cudaStream_t s, double bp)
{
  constexpr int W = Pack<T>::W;
  const int64_t total = A.n * (int64_t) (ld / W);
  const int grid = (int) std::max<int64_t> (1, std::min<int64_t> (
      (int64_t) num_sms () * 8, (total + 255) / 256));
  k_cheb_tail<T><<<grid, 256, 0, s>>> (A.n, ld, zdinv<T> (A), X, R, D, (T) a,
                                       (T) b, first, bp != 0. ? 1 : 0, (T) bp);
  LGH_LAUNCH_CHECK ();
  return 0;
}

template int launch_cheb_tail<double> (const Csr &, double *, const double *,
                                       const double *, int, double, double,
                                       int, cudaStream_t, double);
template int launch_cheb_tail<float> (const Csr &, float *, const float *,
                                      const float *, int, double, double, int,
                                      cudaStream_t, double);

template int launch_cheb_step<double> (const Csr &, double *, const double *,
                                       double *, const double *, double *,
                                       int, double, double, int, cudaStream_t,
                                       double);
template int launch_cheb_step<float> (const Csr &, float *, const float *,
                                      float *, const float *, float *, int,
                                      double, double, int, cudaStream_t, double);

/* per-column ||D^{-1}(S B - Z X)||, ||D^{-1} S B|| ; optional R output */
template <typename TO>
int
zresid_launch (const Csr &Z, int64_t n, int w, const double *Bm, int ldb,
               const double *rs_in, const double *X, int ldx, TO *Rout,
               int ldr, double *out_r, double *out_b, double *partA,
               double *partB, unsigned *counter, int nblocks, cudaStream_t s)
{
  const int ld = round_ld (w);
  const int nvec = ld / 2;
  int glog, ch;
  row_group_shape (nvec, glog, ch, Z.max_row_nnz);
  const int grid = std::min (row_grid (n, glog), nblocks);
  const int smem = zs_smem_bytes (glog, ld);
  ZK zk{ Z.n, Z.rowptr, Z.colidx };
  ZS_DISPATCH (ch, {
    auto kf = k_zresid<TO, CH_>;
    set_smem_attr (kf, smem);
    kf<<<fit_grid (kf, grid, ZS_THREADS, smem), ZS_THREADS, smem, s>>> (zk, Z.vals, Z.dinv, Bm, ldb, rs_in, X,
                                       ldx, Rout, ldr, nvec, glog, w, partA,
                                       partB, counter, out_r, out_b);
  });
  LGH_LAUNCH_CHECK ();
  return 0;
}

template int zresid_launch<double> (const Csr &, int64_t, int, const double *,
                                    int, const double *, const double *, int,
                                    double *, int, double *, double *,
                                    double *, double *, unsigned *, int,
                                    cudaStream_t);
template int zresid_launch<float> (const Csr &, int64_t, int, const double *,
                                   int, const double *, const double *, int,
                                   float *, int, double *, double *, double *,
                                   double *, unsigned *, int, cudaStream_t);

int
zsolve_residual_norms (const Csr &Z, int64_t n, int w, const double *Bm,
                       int ldb, const double *X, int ldx, double *out,
                       cudaStream_t s)
{
  const int ld = round_ld (w);
  DBuf<double> pa, pb;
  DBuf<unsigned> cnt;
  const int nb = num_sms () * 8;
  LGH_TRY (pa.alloc ((size_t) ld * nb));
  LGH_TRY (pb.alloc ((size_t) ld * nb));
  LGH_TRY (cnt.alloc (4));
  LGH_CUDA (cudaMemsetAsync (cnt.p, 0, 4 * sizeof (unsigned), s));
  LGH_TRY (zresid_launch<double> (Z, n, w, Bm, ldb, nullptr, X, ldx,
                                  (double *) nullptr, 0, out, nullptr, pa.p,
                                  pb.p, cnt.p, nb, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}


} /* namespace lgh */
