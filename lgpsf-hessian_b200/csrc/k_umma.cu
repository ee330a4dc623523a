/* k_umma.cu -- the many-shift Woodbury combination of a mixed-precision
 * object on the fifth-generation tensor cores (tcgen05, TMA, TMEM).
 *
 * The same product as k_shift_combine (k_gemm.cu),
 *   out[:, J] = fc[si] Y0[:, j] + W (g[:, si] .* C[:, j]),  J = si m + j,
 * for objects built in mixed precision (FP32 tall blocks, FP64 small
 * dense core): the n x (nshift m) x kept GEMM runs in TF32 with FP32
 * accumulation, three passes per product (hi.hi + hi.lo + lo.hi of the
 * operands split as x = hi + lo, each part a TF32 value), which keeps the
 * product at about FP32 accuracy; the coefficients g, C, the f(c) y0 term
 * and the output stay FP64.
 *
 * Structure of one CTA (128 threads, one output tile of 128 rows x TN
 * columns):
 *   - the split operands live in global memory K-major (A: n x kpad from
 *     W, once per object; B: columns x kpad from g .* C, once per call),
 *     kpad a multiple of 32;
 *   - thread 0 drives an NS-stage pipeline (NS = 2 with one CTA per SM,
 *     or NS = 1 with two or three CTAs per SM that overlap one another's
 *     loads, MMAs and epilogues): TMA tile loads
 *     (cp.async.bulk.tensor.2d, 128-byte swizzle, no multicast) of 32 K
 *     values of A_hi, A_lo, B_hi, B_lo into a stage, completing on the
 *     stage's mbarrier; then 3 x 4 tcgen05.mma kind::tf32 (M = 128,
 *     N = TN, K = 8 each) from that stage into the TMEM accumulator, and a
 *     tcgen05.commit that frees the stage when those MMAs are done;
 *   - after the last commit every warp reads its 32 TMEM lanes (rows)
 *     with tcgen05.ld and writes the caller's column-major output, adding
 *     fc y0 (staged through the freed stage buffer, 32 columns at a time,
 *     with coalesced row loads): for each column the 32 lanes store 32
 *     consecutive doubles.
 * Every mbarrier wait is bounded; a wait that runs out sets *err, the CTA
 * still waits (bounded) for its own MMAs through one final commit, frees
 * its TMEM and returns, and the host reports the error.
 */

#include <cuda.h>

#include <algorithm>

#include "lgh_batch.h"
#include "lgh_internal.h"

namespace lgh
{

namespace
{

constexpr int UM = 128;             /* rows per tile: MMA M, TMEM lanes */
constexpr int UKA = 32;             /* K values per stage: one 128-byte row */
constexpr uint32_t kWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t
su32 (const void *p)
{
  return (uint32_t) __cvta_generic_to_shared (p);
}

__device__ __forceinline__ bool
mbar_try (uint32_t bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile ("{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, p;\n\t}"
                : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}

/* a bounded wait: false when the limit ran out */
__device__ __forceinline__ bool
mbar_wait (uint32_t bar, uint32_t parity)
{
  for (uint32_t it = 0; it < kWaitLimit; it++)
    if (mbar_try (bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void
tma_load_2d (uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
  asm volatile ("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::"
                "complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                :: "r"(dst), "l"((uint64_t) map), "r"(x), "r"(y), "r"(bar)
                : "memory");
}

/* shared-memory matrix descriptor: K-major, 128-byte swizzle, rows of 128
 * bytes in groups of 8 (1024 bytes apart), sm100 descriptor version */
__device__ __forceinline__ uint64_t
sdesc (uint32_t addr)
{
  return (uint64_t) ((addr >> 4) & 0x3FFF) | ((uint64_t) 1 << 16)
         | ((uint64_t) (1024 >> 4) << 32) | ((uint64_t) 1 << 46)
         | ((uint64_t) 2 << 61);
}

__device__ __forceinline__ void
umma_tf32 (uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
  const uint32_t z = 0;
  asm volatile ("{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, "
                "{%5, %6, %7, %8}, p;\n\t}"
                :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc),
                   "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void
umma_commit (uint32_t bar)
{
  asm volatile ("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::"
                "cluster.b64 [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ float
tf32_hi (float x)
{
  uint32_t r;
  asm ("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float (r);
}

template <int TN, int NS>
__global__ void __launch_bounds__ (128, NS == 1 ? 2 : 1)
k_shift_combine_umma (const __grid_constant__ CUtensorMap mAh,
                      const __grid_constant__ CUtensorMap mAl,
                      const __grid_constant__ CUtensorMap mBh,
                      const __grid_constant__ CUtensorMap mBl, int64_t n,
                      int kpad, int m, int nshift,
                      const double *__restrict__ fc,
                      const double *__restrict__ Y0, int ldy0,
                      double *const *__restrict__ out,
                      const int64_t *__restrict__ ldo, int *err)
{
  constexpr uint32_t A_BYTES = UM * 128, B_BYTES = TN * 128;
  constexpr uint32_t STAGE = 2 * A_BYTES + 2 * B_BYTES;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = su32 (smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *const gbase = smem_raw + (base - raw);
  /* barriers: full[NS], empty[NS], done */
  uint64_t *bars = (uint64_t *) (gbase + NS * STAGE);
  uint32_t *holder = (uint32_t *) (bars + 2 * NS + 1);
  int *failed = (int *) (holder + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t row0 = (int64_t) blockIdx.y * UM;
  const int col0 = blockIdx.x * TN;
  const int ncol = nshift * m;
  const uint32_t bfull = su32 (bars), bempty = su32 (bars + NS),
                 bdone = su32 (bars + 2 * NS);

  if (tid == 0) {
    for (int i = 0; i < 2 * NS + 1; i++)
      asm volatile ("mbarrier.init.shared::cta.b64 [%0], 1;"
                    :: "r"(su32 (bars + i)));
    *failed = 0;
    asm volatile ("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile ("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 "
                  "[%0], %1;" :: "r"(su32 (holder)), "r"(TN));
    asm volatile ("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads ();
  asm volatile ("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *holder;

  if (tid == 0) {
    const int natoms = kpad / UKA;
    /* kind::tf32: D F32, A and B TF32, both K-major, N = TN, M = 128 */
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10)
                           | ((uint32_t) (TN >> 3) << 17)
                           | ((uint32_t) (UM >> 4) << 24);
    bool ok = true;
    int issued = 0;          /* atoms whose loads were issued */
    auto load = [&] (int a) {
      const int s = a % NS;
      const uint32_t st = base + s * STAGE;
      asm volatile ("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                    :: "r"(bfull + 8 * s), "r"(STAGE) : "memory");
      tma_load_2d (st, &mAh, a * UKA, (int) row0, bfull + 8 * s);
      tma_load_2d (st + A_BYTES, &mAl, a * UKA, (int) row0, bfull + 8 * s);
      tma_load_2d (st + 2 * A_BYTES, &mBh, a * UKA, col0, bfull + 8 * s);
      tma_load_2d (st + 2 * A_BYTES + B_BYTES, &mBl, a * UKA, col0,
                   bfull + 8 * s);
      issued = a + 1;
    };
    /* the first NS atoms go straight into their stages; atom b + NS
     * reuses atom b's stage once the MMAs of atom b have drained it */
    for (int a = 0; a < NS && a < natoms; a++) load (a);
    for (int b = 0; b < natoms; b++) {
      const int s = b % NS;
      ok = mbar_wait (bfull + 8 * s, (b / NS) & 1);
      if (!ok) break;
      asm volatile ("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t st = base + s * STAGE;
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const uint64_t ah = sdesc (st + 32 * kk);
        const uint64_t al = sdesc (st + A_BYTES + 32 * kk);
        const uint64_t bh = sdesc (st + 2 * A_BYTES + 32 * kk);
        const uint64_t bl = sdesc (st + 2 * A_BYTES + B_BYTES + 32 * kk);
        umma_tf32 (tmem, ah, bh, idesc, (b > 0 || kk > 0) ? 1u : 0u);
        umma_tf32 (tmem, ah, bl, idesc, 1u);
        umma_tf32 (tmem, al, bh, idesc, 1u);
      }
      umma_commit (bempty + 8 * s);
      if (b + NS < natoms) {
        ok = mbar_wait (bempty + 8 * s, (b / NS) & 1);
        if (!ok) break;
        load (b + NS);
      }
    }
    if (!ok) {
      *failed = 1;
      atomicExch (err, 1);
      /* loads still in flight complete on their stage barriers */
      for (int b = std::max (0, issued - NS); b < issued; b++)
        mbar_wait (bfull + 8 * (b % NS), (b / NS) & 1);
    }
    /* one commit after every MMA issued: the accumulator is final (or,
     * after a failure, no MMA is in flight) when it arrives */
    umma_commit (bdone);
  }
  __syncwarp ();
  const bool done = mbar_wait (bdone, 0);
  asm volatile ("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!done) {
    atomicExch (err, 2);
    *failed = 1;
  }
  __syncthreads ();
  /* uniform over the CTA: the TMEM loads below need converged warps */
  if (*failed == 0) {
    const int64_t i = row0 + warp * 32 + lane;
    double *const o = *out;
    const int64_t ld = *ldo;
    /* the stage buffer is free once the last MMA is done: each 32-column
     * chunk's y0 values (128 rows, row stride 33 doubles against bank
     * conflicts) are staged there with coalesced row loads, lane = column */
    double *const sy = (double *) gbase;
    for (int q0 = 0; q0 < TN; q0 += 32) {
      {
        const int Jl = col0 + q0 + lane;
        const int jl = Jl < ncol ? Jl - (Jl / m) * m : 0;
        for (int r = warp; r < UM; r += 4) {
          const int64_t ii = row0 + r;
          sy[r * 33 + lane] = (ii < n && Jl < ncol) ? Y0[ii * ldy0 + jl] : 0.;
        }
      }
      __syncthreads ();
      uint32_t v[32];
      const uint32_t ta = tmem + ((uint32_t) (warp * 32) << 16) + (uint32_t) q0;
      asm volatile ("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, "
                    "%24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]),
                      "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                      "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                      "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
                      "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                      "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(ta));
      asm volatile ("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (i < n) {
        const double *yr = sy + (warp * 32 + lane) * 33;
#pragma unroll
        for (int q = 0; q < 32; q++) {
          const int J = col0 + q0 + q;
          if (J < ncol) {
            const int si = J / m;
            o[i + (int64_t) J * ld] = (double) __uint_as_float (v[q])
                                      + fc[si] * yr[q];
          }
        }
      }
      __syncthreads ();
    }
  }
  asm volatile ("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads ();
  if (warp == 0)
    asm volatile ("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                  :: "r"(tmem), "r"(TN));
}

/* A = W split into TF32 parts: Ah[i][k] + Al[i][k] = W[i][k] (k < kept),
 * zero for kept <= k < kpad */
__global__ void
k_split_rows (int64_t n, int kept, int kpad, const double *__restrict__ W,
              int ldw, float *__restrict__ Ah, float *__restrict__ Al)
{
  const int64_t total = n * kpad;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / kpad;
    const int k = (int) (e - i * kpad);
    const double w = k < kept ? W[i * ldw + k] : 0.;
    const float h = tf32_hi ((float) w);
    Ah[e] = h;
    Al[e] = (float) (w - (double) h);
  }
}

/* B[J][k] = g[k + si kept] C[k + j kept] split into TF32 parts, J < ncolp
 * (zero past nshift m columns and past kept) */
__global__ void
k_split_coef (int kept, int kpad, int m, int nshift, int ncolp,
              const double *__restrict__ g, const double *__restrict__ C,
              float *__restrict__ Bh, float *__restrict__ Bl)
{
  const int64_t total = (int64_t) ncolp * kpad;
  const int ncol = nshift * m;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int J = (int) (e / kpad);
    const int k = (int) (e - (int64_t) J * kpad);
    double b = 0.;
    if (J < ncol && k < kept) {
      const int si = J / m, j = J - si * m;
      b = g[k + (size_t) si * kept] * C[k + (size_t) j * kept];
    }
    const float h = tf32_hi ((float) b);
    Bh[e] = h;
    Bl[e] = (float) (b - (double) h);
  }
}

typedef CUresult (*encode_fn) (CUtensorMap *, CUtensorMapDataType, cuuint32_t,
                               void *, const cuuint64_t *, const cuuint64_t *,
                               const cuuint32_t *, const cuuint32_t *,
                               CUtensorMapInterleave, CUtensorMapSwizzle,
                               CUtensorMapL2promotion,
                               CUtensorMapFloatOOBfill);

encode_fn
encoder ()
{
  static encode_fn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint ("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                 &q) == cudaSuccess
        && q == cudaDriverEntryPointSuccess)
      fn = (encode_fn) p;
  }
  return fn;
}

/* a K-major FP32 operand (rows x kpad, row pitch kpad floats) in boxes of
 * 32 K values x box_rows rows, 128-byte swizzle */
int
encode_kmajor (CUtensorMap *map, const float *base, int64_t rows, int kpad,
               int box_rows)
{
  encode_fn fn = encoder ();
  LGH_CHECK (fn != nullptr, LGH_ERR_SUP, "tensor maps unavailable (driver)");
  LGH_CHECK ((uintptr_t) base % 16 == 0 && kpad % UKA == 0, LGH_ERR_ARG_WRONG,
             "tensor map: operand not aligned");
  const cuuint64_t dims[2] = { (cuuint64_t) kpad, (cuuint64_t) rows };
  const cuuint64_t strides[1] = { (cuuint64_t) kpad * 4 };
  const cuuint32_t box[2] = { (cuuint32_t) UKA, (cuuint32_t) box_rows };
  const cuuint32_t estr[2] = { 1, 1 };
  const CUresult r = fn (map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *) base,
                         dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  LGH_CHECK (r == CUDA_SUCCESS, LGH_ERR_GPU, "cuTensorMapEncodeTiled: %d",
             (int) r);
  return 0;
}

template <int TN, int NS>
constexpr int
umma_smem ()
{
  return NS * (2 * UM * 128 + 2 * TN * 128) + 64 + 1024;
}

template <int TN, int NS>
int
launch_umma_shape (const CUtensorMap *mp, dim3 grid, int64_t n, int kpad,
                   int m, int nshift, const double *fc, const double *Y0,
                   int ldy0, double *const *out, const int64_t *ldo, int *err,
                   cudaStream_t s)
{
  auto k = k_shift_combine_umma<TN, NS>;
  constexpr int sm = umma_smem<TN, NS> ();
  static bool set = false;
  if (!set) {
    LGH_CUDA (cudaFuncSetAttribute (k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    set = true;
  }
  k<<<grid, 128, sm, s>>> (mp[0], mp[1], mp[2], mp[3], n, kpad, m, nshift, fc,
                           Y0, ldy0, out, ldo, err);
  LGH_LAUNCH_CHECK ();
  return 0;
}

} /* namespace */

bool
umma_supported ()
{
  static int cached = -1;
  if (cached < 0) {
    int dev = 0, major = 0, minor = 0;
    cudaGetDevice (&dev);
    cudaDeviceGetAttribute (&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute (&minor, cudaDevAttrComputeCapabilityMinor, dev);
    cached = (major == 10 && minor == 0 && encoder () != nullptr) ? 1 : 0;
  }
  return cached == 1;
}

int
umma_split_rows (int64_t n, int kept, int kpad, const double *W, int ldw,
                 float *Ah, float *Al, cudaStream_t s)
{
  const int64_t tot = n * kpad;
  const int grid = (int) std::min<int64_t> ((tot + 255) / 256, (int64_t) num_sms () * 16);
  k_split_rows<<<std::max (grid, 1), 256, 0, s>>> (n, kept, kpad, W, ldw, Ah, Al);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
umma_split_coef (int kept, int kpad, int m, int nshift, int ncolp,
                 const double *g, const double *C, float *Bh, float *Bl,
                 cudaStream_t s)
{
  const int64_t tot = (int64_t) ncolp * kpad;
  const int grid = (int) std::min<int64_t> ((tot + 255) / 256, (int64_t) num_sms () * 16);
  k_split_coef<<<std::max (grid, 1), 256, 0, s>>> (kept, kpad, m, nshift, ncolp,
                                                   g, C, Bh, Bl);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
umma_encode (UmmaMaps *M, const float *Ah, const float *Al, int64_t n,
             const float *Bh, const float *Bl, int ncolp, int kpad, int tn)
{
  static_assert (sizeof (UmmaMaps::raw) >= 4 * sizeof (CUtensorMap), "maps");
  CUtensorMap *mp = (CUtensorMap *) M->raw;
  LGH_TRY (encode_kmajor (mp + 0, Ah, n, kpad, UM));
  LGH_TRY (encode_kmajor (mp + 1, Al, n, kpad, UM));
  LGH_TRY (encode_kmajor (mp + 2, Bh, ncolp, kpad, tn));
  LGH_TRY (encode_kmajor (mp + 3, Bl, ncolp, kpad, tn));
  M->tn = tn;
  return 0;
}

int
launch_shift_combine_umma (const UmmaMaps &M, int stages, int64_t n, int kpad,
                           int m, int nshift, const double *fc,
                           const double *Y0, int ldy0, double *const *out,
                           const int64_t *ldo, int *err, cudaStream_t s)
{
  if (n == 0 || m == 0 || nshift == 0) return 0;
  const CUtensorMap *mp = (const CUtensorMap *) M.raw;
  const int64_t ncol = (int64_t) nshift * m;
  const int64_t rt = (n + UM - 1) / UM;
  LGH_CHECK (rt < 65536 && ncol < INT32_MAX, LGH_ERR_ARG_OUTOFRANGE,
             "tensor-core shift combine: grid too large");
  LGH_CHECK ((M.tn == 128 || M.tn == 256) && (stages == 1 || stages == 2),
             LGH_ERR_ARG_WRONG, "tensor-core shift combine: no such tile");
  const dim3 grid ((unsigned) ((ncol + M.tn - 1) / M.tn), (unsigned) rt);
  if (M.tn == 256)
    return stages == 1
        ? launch_umma_shape<256, 1> (mp, grid, n, kpad, m, nshift, fc, Y0, ldy0, out, ldo, err, s)
        : launch_umma_shape<256, 2> (mp, grid, n, kpad, m, nshift, fc, Y0, ldy0, out, ldo, err, s);
  return stages == 1
      ? launch_umma_shape<128, 1> (mp, grid, n, kpad, m, nshift, fc, Y0, ldy0, out, ldo, err, s)
      : launch_umma_shape<128, 2> (mp, grid, n, kpad, m, nshift, fc, Y0, ldy0, out, ldo, err, s);
}

} /* namespace lgh */
