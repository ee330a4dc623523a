/* k_strip.cu -- the B product Y = B X in strip form.
 *
 * The reference multiplies B into a block one column at a time (MatMult per
 * column, glr_common_impl.h:325-332).  Row by row on the device (k_spmm.cu)
 * every nonzero (i, j) gathers the whole row X[j, :], so a 220-wide FP64
 * block pulls nnz x 1760 bytes through L1/L2 per product: 84 GB at the
 * 512^2 configuration, for 1.5 GB of algorithmic traffic.  Consecutive rows
 * of a local operator (a kernel matrix on a grid or a well-ordered mesh)
 * share most of their columns, so the strip form groups R consecutive rows
 * and stores, per strip, the union of their column indices with an R-value
 * column of the strip's entries at each (zero where a row has none).  The
 * product then loads each gathered X row once per strip and applies it to
 * the R rows from registers: the gather traffic falls by about the factor
 * (R * nnz per row) / (union per strip), 5x at R = 8 on the 2D kernel
 * matrix, for some padded FMAs.
 *
 * Layout (device):
 *   sptr[s] .. sptr[s+1]   the union entries of strip s (int64)
 *   scol[k]                the column of entry k (int32)
 *   sval[k * R + r]        row r0 + r's value at scol[k] (FP64; sval32 FP32)
 * Building: one group of R lanes per strip merges the R rows' column lists
 * (warp min-reduction over the lanes' current columns; the lanes whose
 * current column is the minimum emit their value and advance).  Each
 * nonzero is emitted exactly once, so the form is exact for any CSR (rows
 * need not be sorted; unsorted rows only lengthen the unions).  Two passes:
 * union lengths, a scan, then the fill.  The strip height R (2, 4 or 8) is
 * chosen per operator from the union lengths by a cost model of the
 * product: padded FMA slots against gathered bytes.
 */

#include <algorithm>

#include "lgh_device.cuh"
#include "lgh_internal.h"
#include "lgh_strip.h"

namespace lgh
{

namespace
{

/* union length (count pass, sval == nullptr) or the fill of each strip of
 * R rows; lanes grouped by R inside a warp, one strip per group */
template <int R>
__global__ void __launch_bounds__ (256)
k_strip_merge (int64_t n, int64_t nstrips, const int64_t *__restrict__ rowptr,
               const int32_t *__restrict__ colidx,
               const double *__restrict__ vals, int64_t *__restrict__ counts,
               const int64_t *__restrict__ sptr, int32_t *__restrict__ scol,
               double *__restrict__ sval, float *__restrict__ sval32,
               unsigned long long *__restrict__ total)
{
  const int lane = threadIdx.x & 31;
  const int sub = lane & (R - 1);
  const unsigned gmask = (R == 32) ? 0xffffffffu
                         : (((1u << R) - 1u) << (lane & ~(R - 1)));
  const int64_t groups_per_cta = blockDim.x / R;
  const int64_t gstride = (int64_t) gridDim.x * groups_per_cta;
  for (int64_t s0 = (int64_t) blockIdx.x * groups_per_cta; s0 < nstrips;
       s0 += gstride) {
    /* every group of the warp runs the loop trip of its own strip; the
     * merge's reductions involve only the group's lanes */
    const int64_t s = s0 + (threadIdx.x / R);
    const bool live = s < nstrips;
    const int64_t row = s * R + sub;
    int64_t k = 0, kend = 0;
    if (live && row < n) {
      k = rowptr[row];
      kend = rowptr[row + 1];
    }
    int64_t pos = (live && sptr) ? sptr[s] : 0;
    int64_t len = 0;
    for (;;) {
      const int cur = (k < kend) ? colidx[k] : INT32_MAX;
      const int m = (int) __reduce_min_sync (gmask, (unsigned) cur);
      if (m == INT32_MAX) break;
      const bool mine = (cur == m);
      if (sval) {
        const double v = mine ? vals[k] : 0.;
        sval[pos * R + sub] = v;
        sval32[pos * R + sub] = (float) v;
        if (sub == 0) scol[pos] = m;
        pos++;
      }
      if (mine) k++;
      len++;
    }
    if (live && !sval && sub == 0) {
      counts[s] = len;
      atomicAdd (total, (unsigned long long) len);
    }
  }
}

/* exclusive scan of counts (one CTA; each thread a contiguous chunk) */
__global__ void __launch_bounds__ (1024)
k_scan_counts (int64_t m, const int64_t *__restrict__ counts,
               int64_t *__restrict__ ptr)
{
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t chunk = (m + blockDim.x - 1) / blockDim.x;
  const int64_t a = (t * chunk < m) ? t * chunk : m;
  const int64_t b = (a + chunk < m) ? a + chunk : m;
  int64_t s = 0;
  for (int64_t i = a; i < b; i++) s += counts[i];
  part[t] = s;
  __syncthreads ();
  if (t == 0) {
    int64_t run = 0;
    for (int i = 0; i < (int) blockDim.x; i++) {
      const int64_t x = part[i];
      part[i] = run;
      run += x;
    }
    ptr[m] = run;
  }
  __syncthreads ();
  int64_t run = part[t];
  for (int64_t i = a; i < b; i++) {
    ptr[i] = run;
    run += counts[i];
  }
}

/* Y (rows r0 .. r0 + R) = strip s times X over the packs of this warp's
 * column slice: lane l owns packs l + 32 h, h < CH, of the slice starting
 * at pack 32 CH blockIdx.y.  The gathers are latency-bound, so the kernel
 * is built for bytes in flight: a warp stages the columns and values of 32
 * union entries in shared memory with coalesced loads, then issues the X
 * gathers of D entries (D CH = 8 packs per lane) before any of their FMAs,
 * reading the values back as shared-memory broadcasts. */
template <typename T, typename TV, int R, int CH>
__global__ void __launch_bounds__ (256, 2)
k_strip_spmm (int64_t n, int64_t nstrips, const int64_t *__restrict__ sptr,
              const int32_t *__restrict__ scol, const TV *__restrict__ sval,
              const T *__restrict__ X, int ldx, T *__restrict__ Y, int ldy,
              int nvec)
{
  constexpr int W = Pack<T>::W;
  constexpr int D = (8 / CH) > 0 ? 8 / CH : 1;
  __shared__ __align__ (16) TV sv_s[8][32 * R];
  __shared__ int sc_s[8][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t s = (int64_t) blockIdx.x * (blockDim.x >> 5) + wid;
  if (s >= nstrips) return;
  const int pbase = blockIdx.y * 32 * CH;
  T acc[R][CH][W];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int h = 0; h < CH; h++)
#pragma unroll
      for (int e = 0; e < W; e++) acc[r][h][e] = T (0);
  const int64_t k0 = sptr[s], k1 = sptr[s + 1];
  TV *sv = sv_s[wid];
  int *sc = sc_s[wid];
  for (int64_t kb = k0; kb < k1; kb += 32) {
    const int cnt = (int) ((k1 - kb) < 32 ? (k1 - kb) : 32);
    /* stage: lane l takes entry kb + l (its column and R values) */
    sc[lane] = lane < cnt ? scol[kb + lane] : 0;
#pragma unroll
    for (int r = 0; r < R; r++)
      sv[lane * R + r] = lane < cnt ? __ldg (sval + (kb + lane) * R + r) : TV (0);
    __syncwarp ();
    for (int t0 = 0; t0 < cnt; t0 += D) {
      Pack<T> x[D][CH];
#pragma unroll
      for (int d = 0; d < D; d++) {
        const int t = t0 + d;
        const T *xr = X + (int64_t) sc[t < cnt ? t : 0] * ldx;
#pragma unroll
        for (int h = 0; h < CH; h++) {
          const int vi = pbase + lane + 32 * h;
          x[d][h] = (t < cnt && vi < nvec) ? ldp_nc (xr + vi * W) : pzero<T> ();
        }
      }
#pragma unroll
      for (int d = 0; d < D; d++) {
        const int t = t0 + d;
        if (t < cnt) {
          /* the entry's R values as 16-byte shared broadcasts */
          T v[R];
          if constexpr (sizeof (TV) == 8) {
#pragma unroll
            for (int r = 0; r < R; r += 2) {
              const double2 u = *reinterpret_cast<const double2 *> (sv + t * R + r);
              v[r] = (T) u.x;
              v[r + 1] = (T) u.y;
            }
          } else if constexpr (R % 4 == 0) {
#pragma unroll
            for (int r = 0; r < R; r += 4) {
              const float4 u = *reinterpret_cast<const float4 *> (sv + t * R + r);
              v[r] = (T) u.x;
              v[r + 1] = (T) u.y;
              v[r + 2] = (T) u.z;
              v[r + 3] = (T) u.w;
            }
          } else {
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = (T) sv[t * R + r];
          }
#pragma unroll
          for (int r = 0; r < R; r++)
#pragma unroll
            for (int h = 0; h < CH; h++)
#pragma unroll
              for (int e = 0; e < W; e++)
                acc[r][h][e] = fma (v[r], x[d][h].v[e], acc[r][h][e]);
        }
      }
    }
    __syncwarp ();
  }
  const int64_t r0 = s * R;
#pragma unroll
  for (int r = 0; r < R; r++) {
    if (r0 + r >= n) break;
    T *yr = Y + (r0 + r) * ldy;
#pragma unroll
    for (int h = 0; h < CH; h++) {
      const int vi = pbase + lane + 32 * h;
      if (vi < nvec) {
        Pack<T> o;
#pragma unroll
        for (int e = 0; e < W; e++) o.v[e] = acc[r][h][e];
        stp (yr + vi * W, o);
      }
    }
  }
}

template <int R>
int
merge_pass (const Csr &A, int64_t nstrips, int64_t *counts,
            unsigned long long *total, const StripForm *S, cudaStream_t s)
{
  const int grid = (int) std::min<int64_t> ((nstrips * R + 255) / 256,
                                            (int64_t) num_sms () * 16);
  if (S)
    k_strip_merge<R><<<std::max (grid, 1), 256, 0, s>>> (
        A.n, nstrips, A.rowptr, A.colidx, A.vals, nullptr, S->sptr, S->scol,
        S->sval, S->sval32, nullptr);
  else
    k_strip_merge<R><<<std::max (grid, 1), 256, 0, s>>> (
        A.n, nstrips, A.rowptr, A.colidx, A.vals, counts, nullptr, nullptr,
        nullptr, nullptr, total);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
merge_any (int R, const Csr &A, int64_t nstrips, int64_t *counts,
           unsigned long long *total, const StripForm *S, cudaStream_t s)
{
  if (R == 2) return merge_pass<2> (A, nstrips, counts, total, S, s);
  if (R == 4) return merge_pass<4> (A, nstrips, counts, total, S, s);
  return merge_pass<8> (A, nstrips, counts, total, S, s);
}

/* modelled cost of one product per block column at strip height R: each
 * union entry costs R FMA slots and one gathered X element; a gathered
 * element costs about as much as kGather FMA slots (on-chip bandwidth
 * against the FP64 FMA rate) */
constexpr double kGather = 12.0;

double
strip_cost (double unions, int R)
{
  return unions * std::max ((double) R, kGather);
}

} /* namespace */

void
strip_free (StripForm &S)
{
  dfree (S.sptr);
  dfree (S.scol);
  dfree (S.sval);
  dfree (S.sval32);
  S = StripForm ();
}

int
strip_build (const Csr &A, int force_R, StripForm &S)
{
  cudaStream_t s = stream ();
  strip_free (S);
  const int64_t n = A.n;
  if (n == 0 || A.nnz == 0) return 0;
  const int cand[3] = { 2, 4, 8 };
  DBuf<unsigned long long> tot;
  LGH_TRY (tot.alloc (4));
  LGH_CUDA (cudaMemsetAsync (tot.p, 0, 4 * sizeof (unsigned long long), s));
  DBuf<int64_t> cnt[3];
  for (int c = 0; c < 3; c++)
    LGH_TRY (cnt[c].alloc ((size_t) (n + cand[c] - 1) / cand[c] + 1));
  int R = force_R;
  if (R <= 0) {
    for (int c = 0; c < 3; c++)
      LGH_TRY (merge_any (cand[c], A, (n + cand[c] - 1) / cand[c], cnt[c].p,
                          tot.p + c, nullptr, s));
    unsigned long long th[3];
    LGH_CUDA (cudaMemcpyAsync (th, tot.p, sizeof (th), cudaMemcpyDeviceToHost, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    double best = 0.;
    for (int c = 0; c < 3; c++) {
      const double cost = strip_cost ((double) th[c], cand[c]);
      if (R <= 0 || cost < best) { best = cost; R = cand[c]; }
    }
  }
  S.R = R;
  S.n = n;
  S.nstrips = (n + R - 1) / R;
  S.nnz = A.nnz;
  const int ci = R == 2 ? 0 : (R == 4 ? 1 : 2);
  int64_t *counts = cnt[ci].p;
  if (force_R > 0)   /* only the forced height was not counted above */
    LGH_TRY (merge_any (R, A, S.nstrips, counts, tot.p + ci, nullptr, s));
  unsigned long long nent = 0;
  LGH_CUDA (cudaMemcpyAsync (&nent, tot.p + ci, sizeof (nent),
                             cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  S.nent = (int64_t) nent;
  LGH_TRY (dalloc ((void **) &S.sptr, (size_t) (S.nstrips + 1) * sizeof (int64_t)));
  LGH_TRY (dalloc ((void **) &S.scol, (size_t) S.nent * sizeof (int32_t) + 16));
  LGH_TRY (dalloc ((void **) &S.sval, (size_t) S.nent * R * sizeof (double) + 16));
  LGH_TRY (dalloc ((void **) &S.sval32, (size_t) S.nent * R * sizeof (float) + 16));
  k_scan_counts<<<1, 1024, 0, s>>> (S.nstrips, counts, S.sptr);
  LGH_LAUNCH_CHECK ();
  LGH_TRY (merge_any (R, A, S.nstrips, nullptr, nullptr, &S, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

template <typename T, typename TV, int R>
static int
strip_dispatch (const StripForm &S, const TV *sval, const T *X, int ldx, T *Y,
                int ldy, int nvec, cudaStream_t s)
{
  /* one warp per strip and slice of 32 CH packs: R x CH = 16 accumulator
   * packs and 8 packs of gathers in flight per lane within 128 registers
   * (two CTAs of 8 warps per SM) */
  constexpr int CH = 16 / R;
  const int slices = (nvec + 32 * CH - 1) / (32 * CH);
  const int64_t ctas = (S.nstrips + 7) / 8;
  LGH_CHECK (ctas < (int64_t) INT32_MAX && slices < 65536, LGH_ERR_ARG_OUTOFRANGE,
             "strip product: grid too large");
  dim3 grid ((unsigned) ctas, (unsigned) slices);
  k_strip_spmm<T, TV, R, CH><<<grid, 256, 0, s>>> (S.n, S.nstrips, S.sptr,
                                                   S.scol, sval, X, ldx, Y,
                                                   ldy, nvec);
  LGH_LAUNCH_CHECK ();
  return 0;
}

template <typename T>
int
launch_strip_spmm (const StripForm &S, const T *X, int ldx, T *Y, int ldy,
                   int w, cudaStream_t s)
{
  constexpr int W = Pack<T>::W;
  LGH_CHECK (ldx % W == 0 && ldy % W == 0 && (uintptr_t) X % 16 == 0
             && (uintptr_t) Y % 16 == 0, LGH_ERR_ARG_WRONG,
             "strip product: blocks must be 16-byte aligned row-major");
  if (S.nstrips == 0 || w == 0) return 0;
  const int nvec = (w + W - 1) / W;
  /* FP32 blocks take the FP32 copy of the values (the mixed form) */
  const T *sv;
  if constexpr (sizeof (T) == 4) sv = S.sval32;
  else sv = S.sval;
  if (S.R == 2) return strip_dispatch<T, T, 2> (S, sv, X, ldx, Y, ldy, nvec, s);
  if (S.R == 4) return strip_dispatch<T, T, 4> (S, sv, X, ldx, Y, ldy, nvec, s);
  return strip_dispatch<T, T, 8> (S, sv, X, ldx, Y, ldy, nvec, s);
}

template int launch_strip_spmm<double> (const StripForm &, const double *, int,
                                        double *, int, int, cudaStream_t);
template int launch_strip_spmm<float> (const StripForm &, const float *, int,
                                       float *, int, int, cudaStream_t);

} /* namespace lgh */
