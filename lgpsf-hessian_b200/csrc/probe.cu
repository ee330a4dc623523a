/* probe.cu -- throughput probes behind the roofline denominators that the
 * measured copy bandwidth and bf16 GEMM rate do not cover: the FP64 and
 * FP32 FMA pipes, the FP64 mma.sync tensor pipe and the L2-resident read
 * bandwidth, each timed with CUDA events on the library's stream.  Each
 * kernel keeps independent accumulator chains in registers and writes one
 * value per thread (into a buffer sized to its grid), so nothing but the
 * measured pipe bounds it.
 */

#include "lgh_internal.h"

namespace lgh
{

namespace
{

template <typename T>
__global__ void
k_probe_fma (T *out, int iters, T a, T b)
{
  T acc[8];
#pragma unroll
  for (int c = 0; c < 8; c++) acc[c] = (T) (threadIdx.x + c);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int c = 0; c < 8; c++) acc[c] = fma (acc[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) s += acc[c];
  out[(size_t) blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void
k_probe_dmma (double *out, int iters)
{
  const double a = 1.0 + threadIdx.x * 1e-9, b = 1.0 - threadIdx.x * 1e-9;
  double c[4][2] = {};
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 4; i++)
      asm volatile ("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 "
                    "{%0, %1}, {%2}, {%3}, {%0, %1};"
                    : "+d"(c[i][0]), "+d"(c[i][1]) : "d"(a), "d"(b));
  }
  double s = 0;
  for (int i = 0; i < 4; i++) s += c[i][0] + c[i][1];
  out[(size_t) blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void
k_probe_read (const double2 *x, size_t n2, double *out, int reps)
{
  double a = 0, b = 0;
  for (int r = 0; r < reps; r++)
    for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n2;
         i += (size_t) gridDim.x * blockDim.x) {
      const double2 v = __ldcg (x + i);
      a += v.x;
      b += v.y;
    }
  out[(size_t) blockIdx.x * blockDim.x + threadIdx.x] = a + b;
}

} /* namespace */

} /* namespace lgh */

using namespace lgh;

/* out[0..3] = FP64 FMA TFLOP/s, FP32 FMA TFLOP/s, FP64 mma.sync TFLOP/s,
 * L2-resident read GB/s (64 MiB buffer) */
extern "C" int
lgh_probe_peaks (double *out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (out, LGH_ERR_ARG_NULL, "lgh_probe_peaks: NULL");
  cudaStream_t s = stream ();
  const int blocks = num_sms () * 8, threads = 256;
  DBuf<double> d;
  DBuf<float> f;
  DBuf<double2> x;
  const size_t n2 = (size_t) 64 * 1024 * 1024 / 16;
  LGH_TRY (d.alloc ((size_t) blocks * threads));
  LGH_TRY (f.alloc ((size_t) blocks * threads));
  LGH_TRY (x.alloc (n2));
  LGH_CUDA (cudaMemsetAsync (x.p, 0, n2 * 16, s));
  cudaEvent_t e0, e1;
  LGH_CUDA (cudaEventCreate (&e0));
  LGH_CUDA (cudaEventCreate (&e1));
  const int iters = 4096;
  const double thr = (double) blocks * threads;
  float ms = 0.f;
  auto timed = [&] (auto launch) -> double {
    launch ();                          /* warm */
    cudaEventRecord (e0, s);
    launch ();
    cudaEventRecord (e1, s);
    cudaEventSynchronize (e1);
    cudaEventElapsedTime (&ms, e0, e1);
    return ms;
  };
  out[0] = 2.0 * thr * iters * 8 / timed ([&] {
    k_probe_fma<double><<<blocks, threads, 0, s>>> (d.p, iters, 1.0000001, 1e-9);
  }) / 1e9;
  out[1] = 2.0 * thr * iters * 8 / timed ([&] {
    k_probe_fma<float><<<blocks, threads, 0, s>>> (f.p, iters, 1.0000001f, 1e-9f);
  }) / 1e9;
  out[2] = 2.0 * 256.0 * 4 * iters * (thr / 32) / timed ([&] {
    k_probe_dmma<<<blocks, threads, 0, s>>> (d.p, iters);
  }) / 1e9;
  out[3] = (double) n2 * 16 * 20 / timed ([&] {
    k_probe_read<<<blocks, threads, 0, s>>> (x.p, n2, d.p, 20);
  }) / 1e6;
  cudaEventDestroy (e0);
  cudaEventDestroy (e1);
  LGH_CUDA (cudaGetLastError ());
  return 0;
}
