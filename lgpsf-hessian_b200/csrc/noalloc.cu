/* noalloc.cu -- the Gram product X^T X without any device allocation.
 *
 * lgh_gram_noalloc has no counterpart in the reference.  It serves callers
 * that must not allocate device memory: applications that carve the whole
 * device memory budget up front (a memory pool, or a fixed partition per
 * tenant) and forbid a library from taking more, where a cudaMalloc in the
 * library would either fail or break the budget, and loops that must not
 * pay cudaMalloc/cudaFree's device-wide synchronisation on every call.
 * It computes the same product as the Gram step of the build (the split-K
 * kernels of k_gemm.cu), but keeps the per-slice partial sums in one
 * file-scope device array of LGH_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB)
 * that is part of the loaded library image, so every GPU that loads the
 * library holds it until the process exits.  Widths with w * w above that
 * size (w > 1024) are rejected with LGH_ERR_ARG_OUTOFRANGE.
 *
 * Set-up: every call looks the array's device address up with
 * cudaGetSymbolAddress on the current device (the first lookup on a device
 * may load the module), so the address stays right across a device reset
 * or a recreated primary context.  The call runs on the library's stream
 * (the legacy default stream) and synchronises it before returning, so it
 * cannot run while any stream capture is active in the process.  Calls
 * share the one array: two calls whose work overlaps on the GPU (calls
 * from different host threads) race on it and must be serialised by the
 * caller.  Each call overwrites every partial it reads, so nothing has to
 * start at zero and the array keeps the last call's partials.
 */

#include "lgh_internal.h"

namespace lgh
{
int launch_gemm_tn_fixed (int64_t n, int m1, int m2, const double *A, int lda,
                          const double *B, int ldb, double *C, int ldc,
                          double *work, int nsplit, cudaStream_t s);
int gemm_tn_splits (int64_t n, int m1, int m2);
}

#define LGH_NOALLOC_SCRATCH_DOUBLES (1L << 20)

/* split-K partial sums of lgh_gram_noalloc (host code must not use this
 * name as a pointer: it stands for the symbol, not a device address) */
static __device__ __align__ (256) double g_gram_scratch[LGH_NOALLOC_SCRATCH_DOUBLES];

extern "C" int
lgh_gram_noalloc (int64_t n, int w, const double *X, int64_t ldx, double *G,
                  int64_t ldg)
{
  using namespace lgh;
  LGH_TRY (ensure_init ());
  LGH_CHECK (X && G, LGH_ERR_ARG_NULL, "lgh_gram_noalloc: NULL argument");
  LGH_CHECK (n >= 1 && w >= 1 && ldx >= w && ldg >= w, LGH_ERR_ARG_SIZ,
             "lgh_gram_noalloc: need n >= 1, w >= 1, ldx >= w, ldg >= w");
  LGH_CHECK ((int64_t) w * w <= LGH_NOALLOC_SCRATCH_DOUBLES, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_gram_noalloc: w = %d exceeds the fixed scratch (w * w must "
             "be <= %ld, i.e. w <= 1024)", w, (long) LGH_NOALLOC_SCRATCH_DOUBLES);
  LGH_CHECK (ldx <= INT32_MAX && ldg <= INT32_MAX, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_gram_noalloc: leading dimension too large");
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress (&p, g_gram_scratch);
  if (e != cudaSuccess || p == nullptr)
    return set_error (LGH_ERR_GPU, "lgh_gram_noalloc: cudaGetSymbolAddress: %s",
                      cudaGetErrorString (e));
  double *scratch = (double *) p;
  int nsplit = gemm_tn_splits (n, w, w);
  const long fit = LGH_NOALLOC_SCRATCH_DOUBLES / ((long) w * w);
  if (nsplit > fit) nsplit = (int) fit;
  cudaStream_t s = stream ();
  LGH_TRY (launch_gemm_tn_fixed (n, w, w, X, (int) ldx, X, (int) ldx, G,
                                 (int) ldg, scratch, nsplit, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}
