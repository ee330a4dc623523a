/* k_spmm.cu -- CSR times row-major block: Y = A X.
 *
 * Replaces the reference's per-column MatMult loop (glr_common_impl.h:
 * 325-332, and MatMatMult in the Chebyshev core, zsolve_impl.h:123-136).
 * A group of G lanes (a power of two <= 32) owns one row; lane l covers the
 * 16-byte vector columns l, l+G, ..., so every nonzero (i, j) gathers the
 * contiguous row segment X[j, :] with coalesced vector loads, reused from
 * L1/L2 by the neighbouring rows of the same CTA.  The group's lanes fetch
 * G (col, val) pairs at once and broadcast them with shuffles.  Each CTA
 * owns a contiguous row range.  HBM bound; algorithmic bytes
 * nnz (s_v + 4) + 8 (N + 1) + 2 N w s_x.
 */

#include <type_traits>

#include "lgh_device.cuh"
#include "lgh_internal.h"

namespace lgh
{

/* the post-smoothing epilogue of MODE 3 (the coefficients of a two-step
 * Chebyshev-Jacobi sequence; dinv the inverse diagonal) */
template <typename T>
struct SpPost
{
  const T *dinv;
  T a, b, bp;
};

/* MODE 0: Y = A X;  1: Y += A X;  2: Y = B - A X;
 * 3: the last two steps of a post-smoothing sequence in one pass, with
 *    X = B = r0 and Y = x (read and written), A = b1 Z D^{-1}:
 *    r1 = r0 - A r0, d0 = (bp dinv_i) r0, x += d0,
 *    x += (b dinv_i) r1 + a d0 (the roundings of the separate first step
 *    and elementwise tail) */
template <typename T, typename TV, int CH, int MODE>
__global__ void __launch_bounds__ (256)
k_spmm (int64_t n, const int64_t *__restrict__ rowptr,
        const int32_t *__restrict__ colidx, const TV *__restrict__ vals,
        const T *__restrict__ X, int ldx, T *__restrict__ Y, int ldy,
        int nvec, int glog, const T *__restrict__ Bm, int ldb, SpPost<T> pp)
{
  constexpr int W = Pack<T>::W;
  const int G = 1 << glog;
  const int lane = threadIdx.x & (G - 1);
  const int group = threadIdx.x >> glog;
  const int ngroups = blockDim.x >> glog;
  const unsigned gmask = (G == 32) ? 0xffffffffu
                         : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  /* row tiles of ngroups rows interleaved over the CTAs (L2 locality of
   * the gathered neighbour rows); the next row's bounds and first G
   * (column, value) pairs are loaded during the current row's gathers */
  const int64_t stride = (int64_t) gridDim.x * ngroups;
  int64_t i = (int64_t) blockIdx.x * ngroups + group;
  int64_t k0 = 0, k1 = 0;
  int mc = 0;
  T mv = T (0);
  if (i < n) {
    k0 = rowptr[i];
    k1 = rowptr[i + 1];
    if (lane < k1 - k0) {
      mc = colidx[k0 + lane];
      mv = (T) vals[k0 + lane];
    }
  }
  for (; i < n; i += stride) {
    const int64_t inx = i + stride;
    int64_t k0n = 0, k1n = 0;
    if (inx < n) {
      k0n = rowptr[inx];
      k1n = rowptr[inx + 1];
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
          mc = colidx[kb + lane];
          mv = (T) vals[kb + lane];
        }
      }
      for (int t = 0; t < cnt; t++) {
        const int c = __shfl_sync (gmask, mc, t, G);
        const T v = __shfl_sync (gmask, mv, t, G);
        const T *xr = X + (int64_t) c * ldx;
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = lane + h * G;
          if (vi < nvec) {
            Pack<T> x = ldp_nc (xr + vi * W);
#pragma unroll
            for (int e = 0; e < W; e++) acc[h][e] = fma (v, x.v[e], acc[h][e]);
          }
        }
      }
    }
    T *yr = Y + i * ldy;
    T bdi = T (0), bpi = T (0);
    if (MODE == 3) {
      const T di = pp.dinv[i];
      bdi = pp.b * di;
      bpi = pp.bp * di;
    }
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        Pack<T> o;
        if (MODE == 3) {
          Pack<T> r0 = ldp (Bm + i * ldb + vi * W);
          o = ldp (yr + vi * W);
#pragma unroll
          for (int e = 0; e < W; e++) {
            const T r1 = r0.v[e] - acc[h][e];
            const T d0 = fma (bpi, r0.v[e], T (0));
            o.v[e] += d0;
            o.v[e] += fma (bdi, r1, pp.a * d0);
          }
        } else if (MODE == 1) {
          Pack<T> y = ldp (yr + vi * W);
#pragma unroll
          for (int e = 0; e < W; e++) o.v[e] = y.v[e] + acc[h][e];
        } else if (MODE == 2) {
          Pack<T> b = ldp (Bm + i * ldb + vi * W);
#pragma unroll
          for (int e = 0; e < W; e++) o.v[e] = b.v[e] - acc[h][e];
        } else {
#pragma unroll
          for (int e = 0; e < W; e++) o.v[e] = acc[h][e];
        }
        stp (yr + vi * W, o);
      }
    }
    k0 = k0n;
    k1 = k1n;
    mc = 0;
    mv = T (0);
    if (inx < n && lane < k1n - k0n) {
      mc = colidx[k0n + lane];
      mv = (T) vals[k0n + lane];
    }
  }
}

/* Scalar form for single vectors and unaligned views (ld not a multiple
 * of the 16-byte vector, or an offset base): G lanes split a row's
 * nonzeros (CSR-vector), reduce with shuffles; columns in a loop. */
template <typename T, typename TV>
__global__ void __launch_bounds__ (256)
k_spmm_scalar (int64_t n, const int64_t *__restrict__ rowptr,
               const int32_t *__restrict__ colidx, const TV *__restrict__ vals,
               const T *__restrict__ X, int ldx, T *__restrict__ Y, int ldy,
               int w)
{
  constexpr int G = 8;
  const int lane = threadIdx.x & (G - 1);
  const unsigned gmask = 0xffu << ((threadIdx.x & 31) & ~(G - 1));
  const int64_t row0 = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int64_t rstride = ((int64_t) gridDim.x * blockDim.x) / G;
  for (int64_t i = row0; i < n; i += rstride) {
    const int64_t k0 = rowptr[i], k1 = rowptr[i + 1];
    for (int c = 0; c < w; c++) {
      T acc = T (0);
      for (int64_t k = k0 + lane; k < k1; k += G)
        acc = fma ((T) vals[k], X[(int64_t) colidx[k] * ldx + c], acc);
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1)
        acc += __shfl_xor_sync (gmask, acc, o, G);
      if (lane == 0) Y[i * ldy + c] = acc;
    }
  }
}

/* lanes per row and vector chunks per lane for a width of nvec vectors */
void
row_group_shape (int nvec, int &glog, int &ch, int kmax)
{
  int g = 1;
  glog = 0;
  while (g < nvec && g < 32) { g <<= 1; glog++; }
  ch = (nvec + g - 1) / g;
  /* a narrow block (one pack per lane) of an operator whose rows fit half
   * the lanes: half the lanes with two packs each keep twice the loads in
   * flight per thread (the smoother, the PCG kernels and the residual at
   * 64 columns measured 8-23% faster; the restriction, whose coarse rows
   * are long, and the prolongation keep kmax = 0) */
  if (kmax > 0 && ch == 1 && g >= 16 && g / 2 >= kmax) {
    g >>= 1;
    glog--;
    ch = (nvec + g - 1) / g;
  }
}

int
row_grid (int64_t n, int glog)
{
  const int rows_per_cta_iter = 256 >> glog;
  int64_t want = (n + rows_per_cta_iter - 1) / rows_per_cta_iter;
  int64_t cap = (int64_t) num_sms () * 8;
  if (want > cap) want = cap;
  return (int) (want > 0 ? want : 1);
}

template <typename T, typename TV>
static int
spmm_dispatch (const Csr &A, const TV *vals, const T *X, int ldx, T *Y,
               int ldy, int w, cudaStream_t s, int mode = 0,
               const T *Bm = nullptr, int ldb = 0,
               SpPost<T> pp = SpPost<T>{ nullptr, T (0), T (0), T (0) })
{
  constexpr int W = Pack<T>::W;
  const int MAXCH = 10;
  const bool vec_ok = (ldx % W == 0) && (ldy % W == 0)
                      && ((uintptr_t) X % 16 == 0) && ((uintptr_t) Y % 16 == 0)
                      && (mode < 2 || (ldb % W == 0 && (uintptr_t) Bm % 16 == 0));
  if (!vec_ok) {
    if (mode != 0)
      return set_error (LGH_ERR_ARG_WRONG, "spmm: accumulate/residual forms "
                        "need 16-byte aligned row-major blocks");
    int64_t g = (A.n * 8 + 255) / 256;
    if (g > (int64_t) num_sms () * 16) g = (int64_t) num_sms () * 16;
    if (g < 1) g = 1;
    k_spmm_scalar<T, TV><<<(int) g, 256, 0, s>>> (A.n, A.rowptr, A.colidx,
                                                  vals, X, ldx, Y, ldy, w);
    LGH_LAUNCH_CHECK ();
    return 0;
  }
  /* column chunks of at most 32 lanes * MAXCH vectors */
  for (int c0 = 0; c0 < w; c0 += 32 * MAXCH * W) {
    const int wc = (w - c0) < 32 * MAXCH * W ? (w - c0) : 32 * MAXCH * W;
    const int nvec = (wc + W - 1) / W;
    int glog, ch;
    row_group_shape (nvec, glog, ch, mode >= 2 ? A.max_row_nnz : 0);
    const int grid = row_grid (A.n, glog);
    const T *Xc = X + c0;
    T *Yc = Y + c0;
    const T *Bc = Bm ? Bm + c0 : nullptr;
#define LGH_SPMM_MODE(C, M)                                                  \
  k_spmm<T, TV, C, M><<<fit_grid (k_spmm<T, TV, C, M>, grid, 256, 0), 256,   \
                        0, s>>> (A.n, A.rowptr, A.colidx, vals, Xc, ldx, Yc, \
                                 ldy, nvec, glog, Bc, ldb, pp)
#define LGH_SPMM_CASE(C)                                                     \
  case C:                                                                    \
    if (mode == 0) LGH_SPMM_MODE (C, 0);                                     \
    else if (mode == 1) LGH_SPMM_MODE (C, 1);                                \
    else if (mode == 2) LGH_SPMM_MODE (C, 2);                                \
    else LGH_SPMM_MODE (C, 3);                                               \
    break;
    switch (ch) {
      LGH_SPMM_CASE (1) LGH_SPMM_CASE (2) LGH_SPMM_CASE (3)
      LGH_SPMM_CASE (4) LGH_SPMM_CASE (5) LGH_SPMM_CASE (6)
      LGH_SPMM_CASE (7) LGH_SPMM_CASE (8) LGH_SPMM_CASE (9)
      LGH_SPMM_CASE (10)
    default:
      return set_error (LGH_ERR_SUP, "spmm: unsupported chunking %d", ch);
    }
#undef LGH_SPMM_CASE
#undef LGH_SPMM_MODE
    LGH_LAUNCH_CHECK ();
  }
  return 0;
}

template <>
int
launch_spmm<double> (const Csr &A, const double *X, int ldx, double *Y,
                     int ldy, int w, cudaStream_t s)
{
  return spmm_dispatch<double, double> (A, A.vals, X, ldx, Y, ldy, w, s);
}

template <>
int
launch_spmm<float> (const Csr &A, const float *X, int ldx, float *Y, int ldy,
                    int w, cudaStream_t s)
{
  return spmm_dispatch<float, float> (A, A.vals32, X, ldx, Y, ldy, w, s);
}

/* Y += A X (mode 1) or Y = B - A X (mode 2) on aligned row-major blocks */
template <>
int
launch_spmm_mode<double> (const Csr &A, const double *X, int ldx, double *Y,
                          int ldy, int w, int mode, const double *Bm, int ldb,
                          cudaStream_t s)
{
  return spmm_dispatch<double, double> (A, A.vals, X, ldx, Y, ldy, w, s, mode,
                                        Bm, ldb);
}

template <>
int
launch_spmm_mode<float> (const Csr &A, const float *X, int ldx, float *Y,
                         int ldy, int w, int mode, const float *Bm, int ldb,
                         cudaStream_t s)
{
  return spmm_dispatch<float, float> (A, A.vals32, X, ldx, Y, ldy, w, s, mode,
                                      Bm, ldb);
}

/* The coarse correction and the whole post-smoothing of a two-step
 * Chebyshev-Jacobi sequence in one pass over the fine rows:
 *   xf = x + P xc          (the prolongation, its order and rounding)
 *   r1 = r - F1 r          (F1 = b1 Z D^{-1}, r the post residual)
 *   d0 = (bp dinv_i) r,  xf += d0,  xf += (b dinv_i) r1 + a d0.
 * Each row is owned by a group of G lanes as in k_spmm; the next row's
 * bounds and first (column, value) chunks of both operators load during
 * the current row's gathers. */
template <typename T, int CH>
__global__ void __launch_bounds__ (256)
k_post_prolong (int64_t n, const int64_t *__restrict__ frp,
                const int32_t *__restrict__ fci, const T *__restrict__ fv,
                const int64_t *__restrict__ prp,
                const int32_t *__restrict__ pci, const T *__restrict__ pv,
                const T *__restrict__ Rr, const T *__restrict__ Xc,
                T *__restrict__ X, int ld, int nvec, int glog, SpPost<T> pp)
{
  constexpr int W = Pack<T>::W;
  const int G = 1 << glog;
  const int lane = threadIdx.x & (G - 1);
  const int group = threadIdx.x >> glog;
  const int ngroups = blockDim.x >> glog;
  const unsigned gmask = (G == 32) ? 0xffffffffu
                         : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
  const int64_t stride = (int64_t) gridDim.x * ngroups;
  int64_t i = (int64_t) blockIdx.x * ngroups + group;
  int64_t k0 = 0, k1 = 0, q0 = 0, q1 = 0;
  int mc = 0, pc = 0;
  T mv = T (0), pw = T (0);
  if (i < n) {
    k0 = frp[i];
    k1 = frp[i + 1];
    q0 = prp[i];
    q1 = prp[i + 1];
    if (lane < k1 - k0) {
      mc = fci[k0 + lane];
      mv = fv[k0 + lane];
    }
    if (lane < q1 - q0) {
      pc = pci[q0 + lane];
      pw = pv[q0 + lane];
    }
  }
  for (; i < n; i += stride) {
    const int64_t inx = i + stride;
    int64_t k0n = 0, k1n = 0, q0n = 0, q1n = 0;
    if (inx < n) {
      k0n = frp[inx];
      k1n = frp[inx + 1];
      q0n = prp[inx];
      q1n = prp[inx + 1];
    }
    /* the prolongation row: (P xc)_i, then xf = x_i + (P xc)_i */
    T xf[CH][W];
#pragma unroll
    for (int h = 0; h < CH; h++)
#pragma unroll
      for (int e = 0; e < W; e++) xf[h][e] = T (0);
    for (int64_t kb = q0; kb < q1; kb += G) {
      const int cnt = (int) ((q1 - kb) < G ? (q1 - kb) : G);
      if (kb != q0) {
        pc = 0;
        pw = T (0);
        if (lane < cnt) {
          pc = pci[kb + lane];
          pw = pv[kb + lane];
        }
      }
      for (int t = 0; t < cnt; t++) {
        const int c = __shfl_sync (gmask, pc, t, G);
        const T v = __shfl_sync (gmask, pw, t, G);
        const T *xr = Xc + (int64_t) c * ld;
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = lane + h * G;
          if (vi < nvec) {
            Pack<T> x = ldp_nc (xr + vi * W);
#pragma unroll
            for (int e = 0; e < W; e++) xf[h][e] = fma (v, x.v[e], xf[h][e]);
          }
        }
      }
    }
    T *xi = X + i * ld;
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        Pack<T> x = ldp (xi + vi * W);
#pragma unroll
        for (int e = 0; e < W; e++) xf[h][e] = x.v[e] + xf[h][e];
      }
    }
    /* the first step's product F1 r */
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
          mc = fci[kb + lane];
          mv = fv[kb + lane];
        }
      }
      for (int t = 0; t < cnt; t++) {
        const int c = __shfl_sync (gmask, mc, t, G);
        const T v = __shfl_sync (gmask, mv, t, G);
        const T *rr = Rr + (int64_t) c * ld;
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = lane + h * G;
          if (vi < nvec) {
            Pack<T> r = ldp_nc (rr + vi * W);
#pragma unroll
            for (int e = 0; e < W; e++) acc[h][e] = fma (v, r.v[e], acc[h][e]);
          }
        }
      }
    }
    /* the next row's first chunks, behind this row's gathers */
    mc = pc = 0;
    mv = pw = T (0);
    if (inx < n) {
      if (lane < k1n - k0n) {
        mc = fci[k0n + lane];
        mv = fv[k0n + lane];
      }
      if (lane < q1n - q0n) {
        pc = pci[q0n + lane];
        pw = pv[q0n + lane];
      }
    }
    const T di = pp.dinv[i];
    const T bdi = pp.b * di, bpi = pp.bp * di;
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = lane + h * G;
      if (vi < nvec) {
        Pack<T> r0 = ldp (Rr + i * ld + vi * W);
        Pack<T> o;
#pragma unroll
        for (int e = 0; e < W; e++) {
          const T r1 = r0.v[e] - acc[h][e];
          const T d0 = fma (bpi, r0.v[e], T (0));
          o.v[e] = xf[h][e] + d0;
          o.v[e] += fma (bdi, r1, pp.a * d0);
        }
        stp (xi + vi * W, o);
      }
    }
    k0 = k0n;
    k1 = k1n;
    q0 = q0n;
    q1 = q1n;
  }
}

template <typename T>
static const T *
mode_vals (const Csr &A)
{
  if constexpr (std::is_same<T, double>::value) return A.vals;
  else return A.vals32;
}

/* the post-smoothing finish (MODE 3): F1 = b1 Z D^{-1} (values
 * fl(b1 vd_ij)), R0 the residual before the first step, X the iterate */
template <typename T>
int
launch_spmm_cheb_post (const Csr &F1, const T *R0, T *X, int ld, int w,
                       const T *dinv, double a, double b, double bp,
                       cudaStream_t s)
{
  if (mode_vals<T> (F1) == nullptr || dinv == nullptr)
    return set_error (LGH_ERR_ARG_WRONG, "spmm: post-smoothing needs values "
                      "and the inverse diagonal");
  return spmm_dispatch<T, T> (F1, mode_vals<T> (F1), R0, ld, X, ld, w, s, 3,
                              R0, ld, SpPost<T>{ dinv, (T) a, (T) b, (T) bp });
}

template int launch_spmm_cheb_post<double> (const Csr &, const double *,
                                            double *, int, int, const double *,
                                            double, double, double,
                                            cudaStream_t);
template int launch_spmm_cheb_post<float> (const Csr &, const float *, float *,
                                           int, int, const float *, double,
                                           double, double, cudaStream_t);

/* the coarse correction and post-smoothing in one pass (k_post_prolong):
 * F1 = b1 Z D^{-1}, R the post residual, P the prolongation, Xc the
 * coarse correction (ld columns each) */
template <typename T>
int
launch_post_prolong (const Csr &F1, const Csr &P, const T *R, const T *Xc,
                     T *X, int ld, int w, const T *dinv, double a, double b,
                     double bp, cudaStream_t s)
{
  constexpr int W = Pack<T>::W;
  if (mode_vals<T> (F1) == nullptr || mode_vals<T> (P) == nullptr
      || dinv == nullptr || P.n != F1.n)
    return set_error (LGH_ERR_ARG_WRONG, "post-prolong: operators");
  if (ld % W || (uintptr_t) R % 16 || (uintptr_t) Xc % 16 || (uintptr_t) X % 16
      || w > 32 * 10 * W)
    return set_error (LGH_ERR_ARG_WRONG, "post-prolong: needs 16-byte aligned "
                      "row-major blocks of at most %d columns", 32 * 10 * W);
  const int nvec = (w + W - 1) / W;
  int glog, ch;
  row_group_shape (nvec, glog, ch, F1.max_row_nnz);
  const int grid = row_grid (F1.n, glog);
  const SpPost<T> pp{ dinv, (T) a, (T) b, (T) bp };
#define LGH_PP_CASE(C)                                                       \
  case C:                                                                    \
    k_post_prolong<T, C><<<fit_grid (k_post_prolong<T, C>, grid, 256, 0),    \
                           256, 0, s>>> (F1.n, F1.rowptr, F1.colidx,         \
                                         mode_vals<T> (F1), P.rowptr,        \
                                         P.colidx, mode_vals<T> (P), R, Xc,  \
                                         X, ld, nvec, glog, pp);             \
    break;
  switch (ch) {
    LGH_PP_CASE (1) LGH_PP_CASE (2) LGH_PP_CASE (3) LGH_PP_CASE (4)
    LGH_PP_CASE (5) LGH_PP_CASE (6) LGH_PP_CASE (7) LGH_PP_CASE (8)
    LGH_PP_CASE (9) LGH_PP_CASE (10)
  default:
    return set_error (LGH_ERR_SUP, "post-prolong: unsupported chunking %d", ch);
  }
#undef LGH_PP_CASE
  LGH_LAUNCH_CHECK ();
  return 0;
}

template int launch_post_prolong<double> (const Csr &, const Csr &,
                                          const double *, const double *,
                                          double *, int, int, const double *,
                                          double, double, double,
                                          cudaStream_t);
template int launch_post_prolong<float> (const Csr &, const Csr &,
                                         const float *, const float *, float *,
                                         int, int, const float *, double,
                                         double, double, cudaStream_t);

} /* namespace lgh */
