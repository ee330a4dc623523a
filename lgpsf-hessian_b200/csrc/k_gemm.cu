/* k_gemm.cu -- tall-skinny dense products on row-major blocks, FP64
 * accumulation (the plain form's DGEMMs):
 *
 *   gemm_tn  C = A^T B over n rows: the Gram X^T X (glr_common_impl.h:
 *            340-366), the projection Q^T Y (:469-489), U^T X (:825-855),
 *            BCGS2 coefficients (glr_scalapack_impl.h:178).  64 x 64 output
 *            tiles, split over n into slices whose partial tiles are summed
 *            in a fixed order (deterministic), optional symmetrisation
 *            T = (C + C^T)/2 in the same pass (glr_common_impl.h:490-494).
 *   gemm_nn  Y = alpha X M + beta Y0 with a small column-major M: the
 *            triangular update X L^{-T} of CholQR2 (:402), U = Q C_kept
 *            (:567), Y += U W (:876).  64 x 64 tiles, k in steps of 16.
 *
 * Each thread accumulates a 4 x 4 register tile; operands are staged in
 * shared memory with 16-byte vector loads.  These products are O(n ell^2)
 * and bounded by the FP64 (or, for float blocks, FP32) pipe.
 */

#include <algorithm>

#include "lgh_device.cuh"
#include "lgh_internal.h"

namespace lgh
{

constexpr int GB = 64, GK = 16;

template <typename T>
__global__ void __launch_bounds__ (256)
k_gemm_tn_part (int64_t n, int m1, int m2, const T *__restrict__ A, int lda,
                const T *__restrict__ B, int ldb, double *__restrict__ work,
                int64_t kchunk)
{
  __shared__ double As[GK][GB + 1], Bs[GK][GB + 1];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int i0 = blockIdx.x * GB, j0 = blockIdx.y * GB;
  const int64_t kb0 = (int64_t) blockIdx.z * kchunk;
  int64_t kb1 = kb0 + kchunk;
  if (kb1 > n) kb1 = n;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.;
  const int lr = tid >> 4;        /* 0..15 : k row in tile   */
  const int lc = (tid & 15) * 4;  /* 0..60 : 4 columns       */
  for (int64_t k0 = kb0; k0 < kb1; k0 += GK) {
    const int64_t kr = k0 + lr;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int ci = i0 + lc + e, cj = j0 + lc + e;
      As[lr][lc + e] = (kr < kb1 && ci < m1) ? (double) A[kr * lda + ci] : 0.;
      Bs[lr][lc + e] = (kr < kb1 && cj < m2) ? (double) B[kr * ldb + cj] : 0.;
    }
    __syncthreads ();
#pragma unroll
    for (int kk = 0; kk < GK; kk++) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; a++) av[a] = As[kk][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; b++) bv[b] = Bs[kk][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = fma (av[a], bv[b], acc[a][b]);
    }
    __syncthreads ();
  }
  double *wz = work + (size_t) blockIdx.z * m1 * m2;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      if (i < m1 && j < m2) wz[i + (size_t) j * m1] = acc[a][b];
    }
}

__global__ void
k_gemm_tn_reduce (int m1, int m2, int nsplit, const double *__restrict__ work,
                  double *C, int ldc, int sym)
{
  const int64_t total = (int64_t) m1 * m2;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int i = (int) (e % m1), j = (int) (e / m1);
    double s = 0.;
    for (int z = 0; z < nsplit; z++) s += work[(size_t) z * total + e];
    if (sym) {
      double s2 = 0.;
      const int64_t et = (int64_t) j + (int64_t) i * m1;
      for (int z = 0; z < nsplit; z++) s2 += work[(size_t) z * total + et];
      s = 0.5 * (s + s2);
    }
    C[i + (size_t) j * ldc] = s;
  }
}

static int
tn_splits (int64_t n, int m1, int m2)
{
  const int tiles = ((m1 + GB - 1) / GB) * ((m2 + GB - 1) / GB);
  int want = (2 * num_sms () + tiles - 1) / tiles;
  int64_t maxs = (n + 255) / 256;
  if (want > maxs) want = (int) maxs;
  if (want < 1) want = 1;
  if (want > 256) want = 256;
  return want;
}

size_t
gemm_tn_work_elems (int64_t n, int m1, int m2)
{
  return (size_t) tn_splits (n, m1, m2) * m1 * m2;
}

template <typename T>
int
launch_gemm_tn (int64_t n, int m1, int m2, const T *A, int lda, const T *B,
                int ldb, double *C, int ldc, int sym, double *work,
                size_t work_elems, cudaStream_t s)
{
  if (m1 == 0 || m2 == 0) return 0;
  LGH_CHECK (!sym || m1 == m2, LGH_ERR_ARG_SIZ, "gemm_tn: sym needs square");
  const int ns = tn_splits (n, m1, m2);
  LGH_CHECK ((size_t) ns * m1 * m2 <= work_elems, LGH_ERR_ARG_SIZ,
             "gemm_tn: workspace too small");
  int64_t kchunk = (n + ns - 1) / ns;
  kchunk = (kchunk + GK - 1) / GK * GK;
  dim3 grid ((m1 + GB - 1) / GB, (m2 + GB - 1) / GB, ns);
  k_gemm_tn_part<T><<<grid, 256, 0, s>>> (n, m1, m2, A, lda, B, ldb, work,
                                          kchunk);
  LGH_LAUNCH_CHECK ();
  const int64_t total = (int64_t) m1 * m2;
  int rg = (int) std::min<int64_t> ((total + 255) / 256, num_sms () * 8);
  k_gemm_tn_reduce<<<rg, 256, 0, s>>> (m1, m2, ns, work, C, ldc, sym);
  LGH_LAUNCH_CHECK ();
  return 0;
}

/* the same product with an explicit split count and caller-provided
 * partial-sum storage of nsplit * m1 * m2 doubles */
int
launch_gemm_tn_fixed (int64_t n, int m1, int m2, const double *A, int lda,
                      const double *B, int ldb, double *C, int ldc,
                      double *work, int nsplit, cudaStream_t s)
{
  if (m1 == 0 || m2 == 0) return 0;
  if (nsplit < 1) nsplit = 1;
  int64_t kchunk = (n + nsplit - 1) / nsplit;
  kchunk = (kchunk + GK - 1) / GK * GK;
  dim3 grid ((m1 + GB - 1) / GB, (m2 + GB - 1) / GB, nsplit);
  k_gemm_tn_part<double><<<grid, 256, 0, s>>> (n, m1, m2, A, lda, B, ldb,
                                               work, kchunk);
  LGH_LAUNCH_CHECK ();
  const int64_t total = (int64_t) m1 * m2;
  int rg = (int) std::min<int64_t> ((total + 255) / 256, num_sms () * 8);
  k_gemm_tn_reduce<<<rg, 256, 0, s>>> (m1, m2, nsplit, work, C, ldc, 0);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
gemm_tn_splits (int64_t n, int m1, int m2)
{
  return tn_splits (n, m1, m2);
}

template int launch_gemm_tn<double> (int64_t, int, int, const double *, int,
                                     const double *, int, double *, int, int,
                                     double *, size_t, cudaStream_t);
template int launch_gemm_tn<float> (int64_t, int, int, const float *, int,
                                    const float *, int, double *, int, int,
                                    double *, size_t, cudaStream_t);

template <typename T>
__global__ void __launch_bounds__ (256)
k_gemm_nn (int64_t n, int k, int m2, double alpha, const T *__restrict__ X,
           int ldx, const double *__restrict__ M, int ldm, double beta,
           const T *Y0, int ldy0, T *Y, int ldy)
{
  __shared__ double Xs[GB][GK + 1], Ms[GK][GB + 1];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int64_t i0 = (int64_t) blockIdx.x * GB;
  const int j0 = blockIdx.y * GB;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.;
  const int xr = tid >> 2, xk = (tid & 3) * 4;  /* X tile: 64 rows x 16 k */
  const int mj = tid >> 2, mk = (tid & 3) * 4;  /* M tile: 16 k x 64 cols */
  for (int k0 = 0; k0 < k; k0 += GK) {
    const int64_t gi = i0 + xr;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int kk = k0 + xk + e;
      Xs[xr][xk + e] = (gi < n && kk < k) ? (double) X[gi * ldx + kk] : 0.;
      const int gj = j0 + mj, mkk = k0 + mk + e;
      Ms[mk + e][mj] = (gj < m2 && mkk < k) ? M[mkk + (size_t) gj * ldm] : 0.;
    }
    __syncthreads ();
#pragma unroll
    for (int kk = 0; kk < GK; kk++) {
      double xv[4], mv[4];
#pragma unroll
      for (int a = 0; a < 4; a++) xv[a] = Xs[ty + 16 * a][kk];
#pragma unroll
      for (int b = 0; b < 4; b++) mv[b] = Ms[kk][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = fma (xv[a], mv[b], acc[a][b]);
    }
    __syncthreads ();
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int64_t i = i0 + ty + 16 * a;
      const int j = j0 + tx + 16 * b;
      if (i < n && j < m2) {
        double v = alpha * acc[a][b];
        if (beta != 0.) v += beta * (double) Y0[i * ldy0 + j];
        Y[i * ldy + j] = (T) v;
      }
    }
}

template <typename T>
int
launch_gemm_nn (int64_t n, int k, int m2, double alpha, const T *X, int ldx,
                const double *M, int ldm, double beta, const T *Y0, int ldy0,
                T *Y, int ldy, cudaStream_t s)
{
  if (n == 0 || m2 == 0) return 0;
  dim3 grid ((unsigned) ((n + GB - 1) / GB), (unsigned) ((m2 + GB - 1) / GB));
  k_gemm_nn<T><<<grid, 256, 0, s>>> (n, k, m2, alpha, X, ldx, M, ldm, beta,
                                     Y0, ldy0, Y, ldy);
  LGH_LAUNCH_CHECK ();
  return 0;
}

template int launch_gemm_nn<double> (int64_t, int, int, double,
                                     const double *, int, const double *, int,
                                     double, const double *, int, double *,
                                     int, cudaStream_t);
template int launch_gemm_nn<float> (int64_t, int, int, double, const float *,
                                    int, const double *, int, double,
                                    const float *, int, float *, int,
                                    cudaStream_t);

} /* namespace lgh */
