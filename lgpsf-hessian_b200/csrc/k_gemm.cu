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
 *   dense_apply  Y = A^{-1} B on the multigrid's dense coarse level.
 *
 * All three run on the FP64 tensor cores: a CTA of 4 warps owns a 64 x 64
 * output tile, each warp a 32 x 32 quarter of 4 x 4 mma.sync m8n8k4 f64
 * tiles; operands are staged k-major in shared memory 16 k-values at a
 * time (rows padded to 68 doubles so that a fragment load touches 16
 * distinct bank pairs), and the next stage is read into registers while
 * the current one is multiplied.  Float blocks (mixed path) are widened to
 * FP64 as they are staged; every product accumulates in FP64.  These
 * products are O(n ell^2) and bounded by the FP64 tensor pipe.
 */

#include <algorithm>

#include "lgh_batch.h"
#include "lgh_device.cuh"
#include "lgh_internal.h"

namespace lgh
{

constexpr int GB = 64, GK = 16;
constexpr int SLD = GB + 4;   /* shared row stride, doubles */

/* one staged k block: As[k][i] (k-major), Bs[k][j]; warp (wm, wn) adds
 * its 32 x 32 quarter.  m8n8k4 f64 fragments: A (8 x 4, row) holds
 * A[lane / 4][lane % 4], B (4 x 8, col) holds B[lane % 4][lane / 4],
 * C holds C[lane / 4][2 (lane % 4) + {0, 1}]. */
__device__ __forceinline__ void
dmma_block (const double (*As)[SLD], const double (*Bs)[SLD], int wm, int wn,
            int lane, double (&acc)[4][4][2])
{
#pragma unroll
  for (int kk = 0; kk < GK; kk += 4) {
    double a[4], b[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      a[t] = As[kk + (lane & 3)][wm * 32 + t * 8 + (lane >> 2)];
      b[t] = Bs[kk + (lane & 3)][wn * 32 + t * 8 + (lane >> 2)];
    }
#pragma unroll
    for (int ti = 0; ti < 4; ti++)
#pragma unroll
      for (int tj = 0; tj < 4; tj++)
        asm volatile ("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
                      "{%0, %1}, {%2}, {%3}, {%0, %1};"
                      : "+d"(acc[ti][tj][0]), "+d"(acc[ti][tj][1])
                      : "d"(a[ti]), "d"(b[tj]));
  }
}

/* the C element of acc[ti][tj][c] inside the CTA tile */
__device__ __forceinline__ int
dmma_row (int wm, int ti, int lane)
{
  return wm * 32 + ti * 8 + (lane >> 2);
}

__device__ __forceinline__ int
dmma_col (int wn, int tj, int c, int lane)
{
  return wn * 32 + tj * 8 + (lane & 3) * 2 + c;
}

/* partial C = A^T B over rows [kb0, kb1) of row-major A (n x m1), B
 * (n x m2), into work[z] (column-major m1 x m2) */
template <typename T>
__global__ void __launch_bounds__ (128)
k_gemm_tn_part (int64_t n, int m1, int m2, const T *__restrict__ A, int lda,
                const T *__restrict__ B, int ldb, double *__restrict__ work,
                int64_t kchunk)
{
  __shared__ double As[GK][SLD], Bs[GK][SLD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int i0 = blockIdx.x * GB, j0 = blockIdx.y * GB;
  const int64_t kb0 = (int64_t) blockIdx.z * kchunk;
  int64_t kb1 = kb0 + kchunk;
  if (kb1 > n) kb1 = n;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.;
  /* staging: thread -> k row (tid / 8), 8 consecutive columns */
  const int lk = tid >> 3, lc = (tid & 7) * 8;
  double ra[8], rb[8];
  auto fetch = [&] (int64_t k0) {
    const int64_t kr = k0 + lk;
    const bool rin = kr < kb1;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int ci = i0 + lc + e, cj = j0 + lc + e;
      ra[e] = (rin && ci < m1) ? (double) A[kr * lda + ci] : 0.;
      rb[e] = (rin && cj < m2) ? (double) B[kr * ldb + cj] : 0.;
    }
  };
  if (kb0 < kb1) fetch (kb0);
  for (int64_t k0 = kb0; k0 < kb1; k0 += GK) {
#pragma unroll
    for (int e = 0; e < 8; e++) {
      As[lk][lc + e] = ra[e];
      Bs[lk][lc + e] = rb[e];
    }
    __syncthreads ();
    if (k0 + GK < kb1) fetch (k0 + GK);   /* next stage behind the mma */
    dmma_block (As, Bs, wm, wn, lane, acc);
    __syncthreads ();
  }
  double *wz = work + (size_t) blockIdx.z * m1 * m2;
#pragma unroll
  for (int ti = 0; ti < 4; ti++)
#pragma unroll
    for (int tj = 0; tj < 4; tj++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int i = i0 + dmma_row (wm, ti, lane), j = j0 + dmma_col (wn, tj, c, lane);
        if (i < m1 && j < m2) wz[i + (size_t) j * m1] = acc[ti][tj][c];
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
  /* about 4 resident 4-warp CTAs per SM over all tiles and slices (the
   * bound of gemm_tn_work_max follows this rule) */
  const int tiles = ((m1 + GB - 1) / GB) * ((m2 + GB - 1) / GB);
  int want = (4 * num_sms () + tiles - 1) / tiles;
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

/* a workspace bound for every shape m1 <= m1max, m2 <= m2max: with t tiles
 * the split count is at most ceil(4 S / t), so splits x tiles <= 4 S + t,
 * and each tile holds at most GB x GB partial sums */
size_t
gemm_tn_work_max (int m1max, int m2max)
{
  const size_t tmax = (size_t) ((m1max + GB - 1) / GB) * ((m2max + GB - 1) / GB);
  return (4 * (size_t) num_sms () + tmax) * GB * GB;
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
  k_gemm_tn_part<T><<<grid, 128, 0, s>>> (n, m1, m2, A, lda, B, ldb, work,
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
  k_gemm_tn_part<double><<<grid, 128, 0, s>>> (n, m1, m2, A, lda, B, ldb,
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

/* Y = alpha X M + beta Y0: X row-major n x k, M column-major k x m2 */
template <typename T>
__global__ void __launch_bounds__ (128)
k_gemm_nn (int64_t n, int k, int m2, double alpha, const T *__restrict__ X,
           int ldx, const double *__restrict__ M, int ldm, double beta,
           const T *Y0, int ldy0, T *Y, int ldy)
{
  __shared__ double As[GK][SLD], Bs[GK][SLD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int64_t i0 = (int64_t) blockIdx.x * GB;
  const int j0 = blockIdx.y * GB;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.;
  /* staging: thread -> tile row / column (tid / 2), 8 consecutive k */
  const int lr = tid >> 1, lk = (tid & 1) * 8;
  double ra[8], rb[8];
  auto fetch = [&] (int k0) {
    const int64_t gi = i0 + lr;
    const int gj = j0 + lr;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int kk = k0 + lk + e;
      ra[e] = (gi < n && kk < k) ? (double) X[gi * ldx + kk] : 0.;
      rb[e] = (gj < m2 && kk < k) ? M[kk + (size_t) gj * ldm] : 0.;
    }
  };
  if (k > 0) fetch (0);
  for (int k0 = 0; k0 < k; k0 += GK) {
#pragma unroll
    for (int e = 0; e < 8; e++) {
      As[lk + e][lr] = ra[e];
      Bs[lk + e][lr] = rb[e];
    }
    __syncthreads ();
    if (k0 + GK < k) fetch (k0 + GK);
    dmma_block (As, Bs, wm, wn, lane, acc);
    __syncthreads ();
  }
#pragma unroll
  for (int ti = 0; ti < 4; ti++)
#pragma unroll
    for (int tj = 0; tj < 4; tj++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int64_t i = i0 + dmma_row (wm, ti, lane);
        const int j = j0 + dmma_col (wn, tj, c, lane);
        if (i < n && j < m2) {
          double v = alpha * acc[ti][tj][c];
          if (beta != 0.) v += beta * (double) Y0[i * ldy0 + j];
          Y[i * ldy + j] = (T) v;
        }
      }
}

/* The Woodbury combination of many shifts in one launch (the batched
 * solve / sample of the shift-independent form x_c = f(c) y0 + W D_c U^T r,
 * glr_common_impl.h:910-929 applied per shift):
 *   out[:, J] = fc[si] Y0[:, j] + W (g[si, :] .* C[:, j]),  J = si m + j,
 * W n x kept row-major (the shift-independent W = Z^{-1} M^{1/2} U), C
 * kept x m column-major (U^T r), g kept x nshift column-major (g[k, si] =
 * f(lam_k + c_si) - f(c_si)), Y0 n x m row-major, out column-major with
 * leading dimension *ldo at *out (the output pointer is read from device
 * memory so that a captured graph serves every call).  One GEMM of n x
 * (nshift m) x kept on the FP64 tensor cores: the shift coefficient is
 * folded into the staging of the B operand, and the epilogue adds f(c) y0
 * and writes the caller's column-major result directly.  Column tiles run
 * fastest, so the CTAs resident at once share a band of W rows in L2. */
/* one staged k block of a BM-row A tile (row stride BM + 4) */
template <int BM>
__device__ __forceinline__ void
dmma_block_rows (const double (*As)[BM + 4], const double (*Bs)[SLD], int wm,
                 int wn, int lane, double (&acc)[4][4][2])
{
#pragma unroll
  for (int kk = 0; kk < GK; kk += 4) {
    double a[4], b[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      a[t] = As[kk + (lane & 3)][wm * 32 + t * 8 + (lane >> 2)];
      b[t] = Bs[kk + (lane & 3)][wn * 32 + t * 8 + (lane >> 2)];
    }
#pragma unroll
    for (int ti = 0; ti < 4; ti++)
#pragma unroll
      for (int tj = 0; tj < 4; tj++)
        asm volatile ("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
                      "{%0, %1}, {%2}, {%3}, {%0, %1};"
                      : "+d"(acc[ti][tj][0]), "+d"(acc[ti][tj][1])
                      : "d"(a[ti]), "d"(b[tj]));
  }
}

/* BM = 64 (4 warps, 2 x 2 quarters of 32 x 32) or 128 (8 warps, 4 x 2) */
template <typename T, int BM>
__global__ void __launch_bounds__ (BM * 2)
k_shift_combine (int64_t n, int kept, int m, int nshift,
                 const T *__restrict__ W, int ldw, const double *__restrict__ C,
                 const double *__restrict__ g, const double *__restrict__ fc,
                 const T *__restrict__ Y0, int ldy0,
                 double *const *__restrict__ out, const int64_t *__restrict__ ldo)
{
  __shared__ double As[GK][BM + 4], Bs[GK][SLD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int ncol = nshift * m;
  const int64_t i0 = (int64_t) blockIdx.y * BM;
  const int j0 = blockIdx.x * GB;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.;
  /* staging: thread -> A tile row tid / 2 (all threads) and B tile column
   * tid / 2 (the first 128 threads), 8 consecutive k each */
  const int lr = tid >> 1, lk = (tid & 1) * 8;
  const bool bthr = lr < GB;
  const int Jr = j0 + lr;
  const bool bcol = bthr && Jr < ncol;
  const int sr = bcol ? Jr / m : 0, jr = bcol ? Jr - sr * m : 0;
  double ra[8], rb[8];
  auto fetch = [&] (int k0) {
    const int64_t gi = i0 + lr;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int kk = k0 + lk + e;
      ra[e] = (gi < n && kk < kept) ? (double) W[gi * ldw + kk] : 0.;
      rb[e] = (bcol && kk < kept)
              ? g[kk + (size_t) sr * kept] * C[kk + (size_t) jr * kept] : 0.;
    }
  };
  if (kept > 0) fetch (0);
  for (int k0 = 0; k0 < kept; k0 += GK) {
#pragma unroll
    for (int e = 0; e < 8; e++) {
      As[lk + e][lr] = ra[e];
      if (bthr) Bs[lk + e][lr] = rb[e];
    }
    __syncthreads ();
    if (k0 + GK < kept) fetch (k0 + GK);
    dmma_block_rows<BM> (As, Bs, wm, wn, lane, acc);
    __syncthreads ();
  }
  double *const o = *out;
  const int64_t ld = *ldo;
#pragma unroll
  for (int tj = 0; tj < 4; tj++)
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int J = j0 + dmma_col (wn, tj, c, lane);
      if (J >= ncol) continue;
      const int si = J / m, j = J - si * m;
      const double f = fc[si];
#pragma unroll
      for (int ti = 0; ti < 4; ti++) {
        const int64_t i = i0 + dmma_row (wm, ti, lane);
        if (i < n)
          o[i + (int64_t) J * ld] = acc[ti][tj][c] + f * (double) Y0[i * ldy0 + j];
      }
    }
}

int
launch_shift_combine_variant (int variant, int64_t n, int kept, int m,
                              int nshift, const double *W, int ldw,
                              const double *C, const double *g,
                              const double *fc, const double *Y0, int ldy0,
                              double *const *out, const int64_t *ldo,
                              cudaStream_t s)
{
  if (n == 0 || m == 0 || nshift == 0) return 0;
  const int BM = variant == 1 ? 128 : 64;
  const int64_t ncol = (int64_t) nshift * m;
  const int64_t rt = (n + BM - 1) / BM;
  LGH_CHECK (ncol < INT32_MAX && rt < 65536, LGH_ERR_ARG_OUTOFRANGE,
             "shift combine: %lld rows x %lld columns exceed the grid",
             (long long) n, (long long) ncol);
  dim3 grid ((unsigned) ((ncol + GB - 1) / GB), (unsigned) rt);
  if (variant == 1)
    k_shift_combine<double, 128><<<grid, 256, 0, s>>> (
        n, kept, m, nshift, W, ldw, C, g, fc, Y0, ldy0, out, ldo);
  else
    k_shift_combine<double, 64><<<grid, 128, 0, s>>> (
        n, kept, m, nshift, W, ldw, C, g, fc, Y0, ldy0, out, ldo);
  LGH_LAUNCH_CHECK ();
  return 0;
}

/* Y = A^{-1} B on the dense coarse level: A^{-1} n0 x n0 column-major,
 * B and Y n0 x ld row-major; columns w .. ld - 1 of Y are set to zero */
template <typename T>
__global__ void __launch_bounds__ (128)
k_dense_apply (int n0, const double *__restrict__ Ainv, const T *__restrict__ B,
               T *__restrict__ Y, int w, int ld)
{
  __shared__ double As[GK][SLD], Bs[GK][SLD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int i0 = blockIdx.x * GB, c0 = blockIdx.y * GB;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.;
  /* staging: thread -> k row (tid / 8), 8 consecutive rows / columns */
  const int lk = tid >> 3, lc = (tid & 7) * 8;
  double ra[8], rb[8];
  auto fetch = [&] (int k0) {
    const int gk = k0 + lk;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int gi = i0 + lc + e, gc = c0 + lc + e;
      ra[e] = (gk < n0 && gi < n0) ? Ainv[gi + (size_t) gk * n0] : 0.;
      rb[e] = (gk < n0 && gc < w) ? (double) B[(size_t) gk * ld + gc] : 0.;
    }
  };
  fetch (0);
  for (int k0 = 0; k0 < n0; k0 += GK) {
#pragma unroll
    for (int e = 0; e < 8; e++) {
      As[lk][lc + e] = ra[e];
      Bs[lk][lc + e] = rb[e];
    }
    __syncthreads ();
    if (k0 + GK < n0) fetch (k0 + GK);
    dmma_block (As, Bs, wm, wn, lane, acc);
    __syncthreads ();
  }
#pragma unroll
  for (int ti = 0; ti < 4; ti++)
#pragma unroll
    for (int tj = 0; tj < 4; tj++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int gi = i0 + dmma_row (wm, ti, lane), gc = c0 + dmma_col (wn, tj, c, lane);
        if (gi < n0 && gc < ld) Y[(size_t) gi * ld + gc] = (gc < w) ? (T) acc[ti][tj][c] : T (0);
      }
}

template <typename T>
int
launch_dense_apply (int n0, const double *Ainv, const T *B, T *Y, int w, int ld,
                    cudaStream_t s)
{
  dim3 grid ((unsigned) ((n0 + GB - 1) / GB), (unsigned) ((ld + GB - 1) / GB));
  k_dense_apply<T><<<grid, 128, 0, s>>> (n0, Ainv, B, Y, w, ld);
  LGH_LAUNCH_CHECK ();
  return 0;
}

template int launch_dense_apply<double> (int, const double *, const double *,
                                         double *, int, int, cudaStream_t);
template int launch_dense_apply<float> (int, const double *, const float *,
                                        float *, int, int, cudaStream_t);

template <typename T>
int
launch_gemm_nn (int64_t n, int k, int m2, double alpha, const T *X, int ldx,
                const double *M, int ldm, double beta, const T *Y0, int ldy0,
                T *Y, int ldy, cudaStream_t s)
{
  if (n == 0 || m2 == 0) return 0;
  dim3 grid ((unsigned) ((n + GB - 1) / GB), (unsigned) ((m2 + GB - 1) / GB));
  k_gemm_nn<T><<<grid, 128, 0, s>>> (n, k, m2, alpha, X, ldx, M, ldm, beta,
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
