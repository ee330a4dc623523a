/* lgh_device.cuh -- device-side helpers shared by the kernels. */

#ifndef LGH_DEVICE_CUH
#define LGH_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

namespace lgh
{

/* 16-byte vector of T: 2 doubles or 4 floats */
template <typename T>
struct __align__ (16) Pack
{
  static constexpr int W = 16 / sizeof (T);
  T v[W];
};

template <typename T>
__device__ __forceinline__ Pack<T>
ldp (const T *p)
{
  return *reinterpret_cast<const Pack<T> *> (p);
}

/* read-only (non-coherent) path: operands not written by this kernel */
template <typename T>
__device__ __forceinline__ Pack<T>
ldp_nc (const T *p)
{
  Pack<T> r;
  if constexpr (sizeof (T) == 8) {
    double2 d = __ldg (reinterpret_cast<const double2 *> (p));
    r.v[0] = d.x; r.v[1] = d.y;
  } else {
    float4 f = __ldg (reinterpret_cast<const float4 *> (p));
    r.v[0] = f.x; r.v[1] = f.y; r.v[2] = f.z; r.v[3] = f.w;
  }
  return r;
}

template <typename T>
__device__ __forceinline__ void
stp (T *p, const Pack<T> &x)
{
  *reinterpret_cast<Pack<T> *> (p) = x;
}

template <typename T>
__device__ __forceinline__ Pack<T>
pzero ()
{
  Pack<T> r;
#pragma unroll
  for (int e = 0; e < Pack<T>::W; e++) r.v[e] = T (0);
  return r;
}

/* contiguous row range of this block: [r0, r1) */
__device__ __forceinline__ void
block_rows (int64_t n, int64_t &r0, int64_t &r1)
{
  int64_t rpb = (n + gridDim.x - 1) / gridDim.x;
  r0 = (int64_t) blockIdx.x * rpb;
  r1 = r0 + rpb;
  if (r1 > n) r1 = n;
  if (r0 > n) r0 = n;
}

/* ---- hashed Gaussian: the reference's lgh_randn_at
 * (glr_common_impl.h:35-73): splitmix64 of (seed, i, j) into a nonzero
 * xorshift64* state, then the polar Box-Muller draw (first of the pair). */
__host__ __device__ __forceinline__ uint64_t
rng_state_at (uint64_t seed, int64_t i, int64_t j)
{
  uint64_t z = seed + 0x9E3779B97F4A7C15ULL * (uint64_t) (i + 1)
               + 0xC2B2AE3D27D4EB4FULL * (uint64_t) (j + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return z ? z : 0x853C49E6748FEA9BULL;
}

__device__ __forceinline__ double
randn_from_state (uint64_t s)
{
  for (;;) {
    uint64_t x;
    double u1, u2, q;
    x = s; x ^= x >> 12; x ^= x << 25; x ^= x >> 27; s = x;
    u1 = (double) ((x * 2685821657736338717ULL) >> 11) / 9007199254740992.0;
    x = s; x ^= x >> 12; x ^= x << 25; x ^= x >> 27; s = x;
    u2 = (double) ((x * 2685821657736338717ULL) >> 11) / 9007199254740992.0;
    u1 = 2. * u1 - 1.;
    u2 = 2. * u2 - 1.;
    /* no fused multiply-add: keep the reference's two rounded products */
    q = __dadd_rn (__dmul_rn (u1, u1), __dmul_rn (u2, u2));
    if (q > 0. && q < 1.) {
      double f = sqrt (__ddiv_rn (-2. * log (q), q));
      return __dmul_rn (u1, f);
    }
  }
}

/* ---- deterministic column reduction across blocks -------------------------
 * Each block writes its per-column partial sums transposed, part[c * nb +
 * blockIdx.x] (nb = gridDim.x); the last block to arrive (atomic ticket)
 * reduces one column per warp in a fixed order (lane-strided sums, then a
 * fixed shuffle tree) and calls fin(c, sum) from lane 0.  Returns true in
 * the last block, after all fin calls; resets the ticket for reuse.      */
__device__ __forceinline__ double
warp_sum (double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync (0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ bool
last_block_ticket (unsigned *counter)
{
  __shared__ bool am_last;
  __threadfence ();
  __syncthreads ();
  if (threadIdx.x == 0) {
    unsigned t = atomicAdd (counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads ();
  if (am_last) __threadfence ();
  return am_last;
}

template <typename Fin>
__device__ __forceinline__ bool
last_block_reduce (const double *part, int ld, unsigned *counter, Fin fin)
{
  if (!last_block_ticket (counter)) return false;
  const int nb = gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int c = warp; c < ld; c += nw) {
    double s = 0.;
    for (int b = lane; b < nb; b += 32) s += __ldcg (part + (size_t) c * nb + b);
    s = warp_sum (s);
    if (lane == 0) fin (c, s);
  }
  __syncthreads ();
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

template <typename Fin>
__device__ __forceinline__ bool
last_block_reduce2 (const double *partA, const double *partB, int ld,
                    unsigned *counter, Fin fin)
{
  if (!last_block_ticket (counter)) return false;
  const int nb = gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int c = warp; c < ld; c += nw) {
    double a = 0., b2 = 0.;
    for (int b = lane; b < nb; b += 32) {
      a += __ldcg (partA + (size_t) c * nb + b);
      b2 += __ldcg (partB + (size_t) c * nb + b);
    }
    a = warp_sum (a);
    b2 = warp_sum (b2);
    if (lane == 0) fin (c, a, b2);
  }
  __syncthreads ();
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

/* Block-level column sums: every thread holds CH packs of partial sums for
 * vector columns v = lane + h*G; red is shared scratch of
 * (blockDim/G) * ld doubles.  Writes part[c * gridDim.x + blockIdx.x].   */
template <typename T, int CH>
__device__ __forceinline__ void
block_colsum_store (const double (&acc)[CH][Pack<T>::W], int lane, int group,
                    int G, int nvec, int ld, double *red, double *part)
{
  constexpr int W = Pack<T>::W;
  const int ngroups = blockDim.x / G;
  __syncthreads ();
#pragma unroll
  for (int h = 0; h < CH; h++) {
    int vi = lane + h * G;
    if (vi < nvec) {
#pragma unroll
      for (int e = 0; e < W; e++) red[group * ld + vi * W + e] = acc[h][e];
    }
  }
  __syncthreads ();
  for (int c = threadIdx.x; c < ld; c += blockDim.x) {
    double s = 0.;
    for (int g = 0; g < ngroups; g++) s += red[g * ld + c];
    part[(size_t) c * gridDim.x + blockIdx.x] = s;
  }
}

/* bounded grid barrier for cooperative launches (co-residency guaranteed
 * by the launch); returns false if the wait ran out (error flag set). */
__device__ __forceinline__ bool
grid_barrier (unsigned *count, unsigned *gen, int *err)
{
  __syncthreads ();
  if (threadIdx.x == 0) {
    volatile unsigned *vgen = gen;
    unsigned g = *vgen;
    __threadfence ();
    unsigned arrived = atomicAdd (count, 1u);
    if (arrived == gridDim.x - 1) {
      *count = 0u;
      __threadfence ();
      atomicAdd (gen, 1u);
    } else {
      long spins = 0;
      while (*vgen == g) {
        if (++spins > (1L << 25)) { atomicExch (err, 1); break; }
        __nanosleep (32);
      }
    }
    __threadfence ();
  }
  __syncthreads ();
  return *((volatile int *) err) == 0;
}

} /* namespace lgh */

#endif /* LGH_DEVICE_CUH */
