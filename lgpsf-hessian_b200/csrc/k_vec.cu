/* k_vec.cu -- elementwise and layout kernels on tall blocks.
 *
 * Row scaling by M^{1/2} (MatDiagonalScale, glr_common_impl.h:322,334;
 * VecPointwiseMult, :1017,1021,1089), layout conversion at the C-ABI
 * boundary (column-major MATDENSE <-> row-major device blocks), precision
 * conversion for the mixed path, and the eigen-residual column norms of
 * the build check (glr_common_impl.h:576-600).  All HBM-streaming.
 */

#include "lgh_device.cuh"
#include "lgh_internal.h"

namespace lgh
{

static int
ew_grid (int64_t total)
{
  int64_t g = (total + 255) / 256;
  int64_t cap = (int64_t) num_sms () * 16;
  return (int) (g < 1 ? 1 : (g < cap ? g : cap));
}

template <typename T>
__global__ void
k_rowscale (int64_t n, int w, const double *scale, const T *X, int ldx, T *Y,
            int ldy)
{
  const int64_t total = n * w;
  for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
       idx < total; idx += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = idx / w;
    const int j = (int) (idx - i * w);
    double sc = scale ? scale[i] : 1.0;
    Y[i * ldy + j] = (T) (sc * (double) X[i * ldx + j]);
  }
}

template <typename T>
int
launch_rowscale (int64_t n, int w, const double *scale, const T *X, int ldx,
                 T *Y, int ldy, cudaStream_t s)
{
  if (n == 0 || w == 0) return 0;
  k_rowscale<T><<<ew_grid (n * w), 256, 0, s>>> (n, w, scale, X, ldx, Y, ldy);
  LGH_LAUNCH_CHECK ();
  return 0;
}
template int launch_rowscale<double> (int64_t, int, const double *,
                                      const double *, int, double *, int,
                                      cudaStream_t);
template int launch_rowscale<float> (int64_t, int, const double *,
                                     const float *, int, float *, int,
                                     cudaStream_t);

template <typename T>
int
launch_copy_block (int64_t n, int w, const T *X, int ldx, T *Y, int ldy,
                   cudaStream_t s)
{
  if (n == 0 || w == 0) return 0;
  LGH_CUDA (cudaMemcpy2DAsync (Y, (size_t) ldy * sizeof (T), X,
                               (size_t) ldx * sizeof (T), (size_t) w * sizeof (T),
                               (size_t) n, cudaMemcpyDeviceToDevice, s));
  return 0;
}
template int launch_copy_block<double> (int64_t, int, const double *, int,
                                        double *, int, cudaStream_t);
template int launch_copy_block<float> (int64_t, int, const float *, int,
                                       float *, int, cudaStream_t);

/* tiled transpose between column-major (ld64) and row-major (ld) */
template <bool TO_ROW>
__global__ void
k_layout (int64_t n, int w, const double *X, int64_t ldx, double *Y,
          int64_t ldy, const double *scale)
{
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t) blockIdx.x * 32;
  const int j0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
  for (int r = ty; r < 32; r += 8) {
    if (TO_ROW) { /* X col-major: X[i + j*ldx]; read along i */
      int64_t i = i0 + tx;
      int j = j0 + r;
      tile[r][tx] = (i < n && j < w) ? X[i + (int64_t) j * ldx] : 0.;
    } else {      /* X row-major: X[i*ldx + j]; read along j */
      int64_t i = i0 + r;
      int j = j0 + tx;
      tile[r][tx] = (i < n && j < w) ? X[i * ldx + j] : 0.;
    }
  }
  __syncthreads ();
  for (int r = ty; r < 32; r += 8) {
    if (TO_ROW) { /* Y row-major: write along j; tile[j][i] */
      int64_t i = i0 + r;
      int j = j0 + tx;
      if (i < n && j < w)
        Y[i * ldy + j] = tile[tx][r] * (scale ? scale[i] : 1.0);
    } else {      /* Y col-major: write along i; tile[i][j] */
      int64_t i = i0 + tx;
      int j = j0 + r;
      if (i < n && j < w)
        Y[i + (int64_t) j * ldy] = tile[tx][r] * (scale ? scale[i] : 1.0);
    }
  }
}

int
launch_colmajor_to_rowmajor (int64_t n, int w, const double *X, int64_t ldx,
                             double *Y, int ldy, const double *scale,
                             cudaStream_t s)
{
  if (n == 0 || w == 0) return 0;
  dim3 grid ((unsigned) ((n + 31) / 32), (unsigned) ((w + 31) / 32));
  k_layout<true><<<grid, dim3 (32, 8), 0, s>>> (n, w, X, ldx, Y, ldy, scale);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
launch_rowmajor_to_colmajor (int64_t n, int w, const double *X, int ldx,
                             double *Y, int64_t ldy, const double *scale,
                             cudaStream_t s)
{
  if (n == 0 || w == 0) return 0;
  dim3 grid ((unsigned) ((n + 31) / 32), (unsigned) ((w + 31) / 32));
  k_layout<false><<<grid, dim3 (32, 8), 0, s>>> (n, w, X, ldx, Y, ldy, scale);
  LGH_LAUNCH_CHECK ();
  return 0;
}

template <typename TI, typename TO>
__global__ void
k_convert (int64_t n, int w, const TI *X, int ldx, TO *Y, int ldy)
{
  const int64_t total = n * w;
  for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
       idx < total; idx += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = idx / w;
    const int j = (int) (idx - i * w);
    Y[i * ldy + j] = (TO) X[i * ldx + j];
  }
}

int
launch_f64_to_f32 (int64_t n, int w, const double *X, int ldx, float *Y,
                   int ldy, cudaStream_t s)
{
  if (n == 0 || w == 0) return 0;
  k_convert<double, float><<<ew_grid (n * w), 256, 0, s>>> (n, w, X, ldx, Y, ldy);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
launch_f32_to_f64 (int64_t n, int w, const float *X, int ldx, double *Y,
                   int ldy, cudaStream_t s)
{
  if (n == 0 || w == 0) return 0;
  k_convert<float, double><<<ew_grid (n * w), 256, 0, s>>> (n, w, X, ldx, Y, ldy);
  LGH_LAUNCH_CHECK ();
  return 0;
}

int
launch_zero_block (int64_t n, int ld, void *Y, size_t elem, cudaStream_t s)
{
  if (n == 0) return 0;
  LGH_CUDA (cudaMemsetAsync (Y, 0, (size_t) n * ld * elem, s));
  return 0;
}

/* || FU[:, j] - lam[j] U[:, j] ||_2, deterministic two-level sum */
template <typename T>
__global__ void
k_resid_norms (int64_t n, int w, const T *FU, int ldf, const T *U, int ldu,
               const double *lam, double *out, double *part, unsigned *counter)
{
  extern __shared__ double red[];
  int64_t r0, r1;
  block_rows (n, r0, r1);
  /* one thread per column (w <= blockDim.x * k), rows of this block */
  for (int c = threadIdx.x; c < w; c += blockDim.x) {
    double acc = 0.;
    const double l = lam[c];
    for (int64_t i = r0; i < r1; i++) {
      double d = (double) FU[i * ldf + c] - l * (double) U[i * ldu + c];
      acc += d * d;
    }
    part[(size_t) c * gridDim.x + blockIdx.x] = acc;
  }
  last_block_reduce (part, w, counter,
                     [&] (int c, double sum) { out[c] = sqrt (sum); });
}

template <typename T>
int
launch_resid_norms (int64_t n, int w, const T *FU, int ldf, const T *U,
                    int ldu, const double *lam, double *out, double *partials,
                    unsigned *counter, cudaStream_t s)
{
  if (w == 0) return 0;
  int grid = num_sms () * 2;
  k_resid_norms<T><<<grid, 256, 0, s>>> (n, w, FU, ldf, U, ldu, lam, out,
                                          partials, counter);
  LGH_LAUNCH_CHECK ();
  return 0;
}
template int launch_resid_norms<double> (int64_t, int, const double *, int,
                                         const double *, int, const double *,
                                         double *, double *, unsigned *,
                                         cudaStream_t);
template int launch_resid_norms<float> (int64_t, int, const float *, int,
                                        const float *, int, const double *,
                                        double *, double *, unsigned *,
                                        cudaStream_t);

__global__ void
k_vec_scale (int64_t n, const double *x, const double *scale, double alpha,
             double *y)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    y[i] = alpha * x[i] * (scale ? scale[i] : 1.0);
}

int
launch_vec_scale (int64_t n, const double *x, const double *scale,
                  double alpha, double *y, cudaStream_t s)
{
  if (n == 0) return 0;
  k_vec_scale<<<ew_grid (n), 256, 0, s>>> (n, x, scale, alpha, y);
  LGH_LAUNCH_CHECK ();
  return 0;
}

__global__ void
k_vec_axpby (int64_t n, double a, const double *x, double b, const double *y,
             double *out)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    out[i] = a * x[i] + b * y[i];
}

int
launch_vec_axpby (int64_t n, double a, const double *x, double b,
                  const double *y, double *out, cudaStream_t s)
{
  if (n == 0) return 0;
  k_vec_axpby<<<ew_grid (n), 256, 0, s>>> (n, a, x, b, y, out);
  LGH_LAUNCH_CHECK ();
  return 0;
}

__global__ void
k_vec_div (int64_t n, const double *x, const double *d, double *y)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    y[i] = x[i] / d[i];
}

int
launch_vec_div (int64_t n, const double *x, const double *d, double *y,
                cudaStream_t s)
{
  if (n == 0) return 0;
  k_vec_div<<<ew_grid (n), 256, 0, s>>> (n, x, d, y);
  LGH_LAUNCH_CHECK ();
  return 0;
}

} /* namespace lgh */
