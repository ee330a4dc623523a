/* k_sketch.cu -- the hashed Gaussian sketch Omega on the device.
 *
 * Omega_ij = lgh_randn_at(seed, i, j) (glr_common_impl.h:59-73, used at
 * :441-443 for the build and glr_scalapack_impl.h:726-729 for the
 * extension, which continues j past ell).  One thread per entry, written
 * straight into the row-major block that feeds the first F-apply; padding
 * columns j in [k, ld) are zeroed.  HBM-write bound: N * ld * s bytes.
 */

#include "lgh_device.cuh"
#include "lgh_internal.h"

namespace lgh
{

template <typename T>
__global__ void
k_sketch (uint64_t seed, int64_t i0, int64_t n, int64_t j0, int k, T *Y,
          int64_t ld)
{
  const int64_t total = n * ld;
  for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
       idx < total; idx += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = idx / ld;
    const int j = (int) (idx - i * ld);
    double v = 0.;
    if (j < k) v = randn_from_state (rng_state_at (seed, i0 + i, j0 + j));
    Y[idx] = (T) v;
  }
}

__global__ void
k_rng_state (uint64_t seed, int64_t n, int64_t j0, int k, uint64_t *S)
{
  const int64_t total = n * (int64_t) k;
  for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
       idx < total; idx += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = idx / k;
    const int j = (int) (idx - i * k);
    S[idx] = rng_state_at (seed, i, j0 + j);
  }
}

static int
grid_for (int64_t total)
{
  int64_t g = (total + 255) / 256;
  int64_t cap = (int64_t) num_sms () * 16;
  return (int) (g < cap ? (g > 0 ? g : 1) : cap);
}

int
launch_sketch (uint64_t seed, int64_t n, int64_t j0, int k, double *Y,
               int ld, cudaStream_t s, int64_t i0)
{
  if (n == 0) return 0;
  k_sketch<double><<<grid_for (n * ld), 256, 0, s>>> (seed, i0, n, j0, k, Y, ld);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
launch_sketch_f32 (uint64_t seed, int64_t n, int64_t j0, int k, float *Y,
                   int ld, cudaStream_t s, int64_t i0)
{
  if (n == 0) return 0;
  k_sketch<float><<<grid_for (n * ld), 256, 0, s>>> (seed, i0, n, j0, k, Y, ld);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
launch_rng_state (uint64_t seed, int64_t n, int64_t j0, int k, uint64_t *S,
                  cudaStream_t s)
{
  if (n == 0 || k == 0) return 0;
  k_rng_state<<<grid_for (n * k), 256, 0, s>>> (seed, n, j0, k, S);
  LGH_LAUNCH_CHECK ();
  return 0;
}

} /* namespace lgh */

extern "C" int
lgh_sketch_rows (uint64_t seed, int64_t i0, int64_t n, int64_t j0, int k,
                 double *Y, int64_t ld)
{
  using namespace lgh;
  LGH_TRY (ensure_init ());
  LGH_CHECK (Y || n == 0, LGH_ERR_ARG_NULL, "lgh_sketch_rows: NULL");
  LGH_CHECK (i0 >= 0 && n >= 0 && j0 >= 0 && k >= 0 && ld >= k,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_sketch_rows: sizes");
  if (n == 0 || ld == 0) return 0;
  cudaStream_t s = stream ();
  k_sketch<double><<<grid_for (n * ld), 256, 0, s>>> (seed, i0, n, j0, k, Y, ld);
  LGH_LAUNCH_CHECK ();
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

