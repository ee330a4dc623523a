/* api_core.cu -- runtime, errors, Mat / Vec handles and the prior object.
 *
 * The prior mirrors struct lgh_prior (glr_common_impl.h:81-94): mass,
 * M^{1/2}, M^{-1/2} (VecSqrtAbs + VecReciprocal, :114-132), and either the
 * user's callbacks (:134-146) or the Mat path (zsolve_impl.h:720-823) whose
 * Z-solves run on the device (zsolve.cu).  Reference counted; destroy is
 * safe in either order with the GLR objects that hold it (:151-168).
 */

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <map>
#include <mutex>

#include "lgh_device.cuh"
#include "lgh_internal.h"
#include "lgh_mg.h"
#include "lgh_objects.h"

namespace lgh
{

/* ---- errors ---------------------------------------------------------- */

static thread_local std::string g_err;
long g_launches = 0;

int
set_error (int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start (ap, fmt);
  vsnprintf (buf, sizeof (buf), fmt, ap);
  va_end (ap);
  g_err = buf;
  if (getenv ("LGH_VERBOSE")) fprintf (stderr, "lgh: error %d: %s\n", code, buf);
  return code;
}

void
clear_error ()
{
  g_err.clear ();
}

/* ---- runtime --------------------------------------------------------- */

static std::mutex g_init_mu;
static int g_inited = 0, g_sms = 148;

int
ensure_init ()
{
  if (g_inited) return 0;
  std::lock_guard<std::mutex> lk (g_init_mu);
  if (g_inited) return 0;
  int dev = 0;
  LGH_CUDA (cudaGetDevice (&dev));
  LGH_CUDA (cudaDeviceGetAttribute (&g_sms, cudaDevAttrMultiProcessorCount, dev));
  g_inited = 1;
  return 0;
}

/* The synchronous C-ABI calls run on the legacy default stream, so work a
 * caller queued on it (or on any blocking stream) is ordered before them. */
cudaStream_t
stream ()
{
  return cudaStreamLegacy;
}

int
num_sms ()
{
  return g_sms;
}

double
wall ()
{
  return std::chrono::duration<double> (
             std::chrono::steady_clock::now ().time_since_epoch ())
      .count ();
}

RuntimeCounters g_rt;

static std::mutex g_rt_mu;

static void
rt_add (double &sec, long &cnt, double dt)
{
  std::lock_guard<std::mutex> lk (g_rt_mu);
  sec += dt;
  cnt++;
}

/* ---- device memory: a caching allocator -----------------------------------
 * cudaFree synchronises the whole device and, for the build's 0.5 GB
 * blocks, took up to 50 ms apiece on some hosts; a job frees ~30 blocks.
 * Freed blocks therefore go to a cache keyed by size, with an event
 * recorded on the library stream after the free; an allocation takes the
 * smallest cached block of at least its size (and at most twice it), after
 * the host has waited for that block's event, so no work still using the
 * block can overlap its next owner on any stream.  The cache keeps at most
 * a third of the device's memory; when cudaMalloc runs out, the cache is
 * released and the allocation retried.  Sizes are rounded up to 2 MiB
 * above 4 MiB (256 B below) so that repeated shapes reuse blocks. */

namespace
{
struct CachedBlock
{
  void *p;
  size_t bytes;
  cudaEvent_t ev;
};
std::mutex g_pool_mu;
std::multimap<size_t, CachedBlock> g_pool;
std::map<void *, size_t> g_live;     /* allocated block -> rounded size */
size_t g_pool_bytes = 0, g_pool_cap = 0;

size_t
pool_round (size_t b)
{
  if (b == 0) b = 256;
  if (b > ((size_t) 4 << 20)) return (b + ((size_t) 2 << 20) - 1) & ~(((size_t) 2 << 20) - 1);
  return (b + 255) & ~(size_t) 255;
}

void
pool_release_all ()
{
  /* caller holds g_pool_mu */
  for (auto &kv : g_pool) {
    cudaEventSynchronize (kv.second.ev);
    cudaEventDestroy (kv.second.ev);
    cudaFree (kv.second.p);
  }
  g_pool.clear ();
  g_pool_bytes = 0;
}
} /* namespace */

size_t
pool_cached_bytes ()
{
  std::lock_guard<std::mutex> lk (g_pool_mu);
  return g_pool_bytes;
}

int
dalloc (void **p, size_t bytes)
{
  const double t0 = wall ();
  const size_t rb = pool_round (bytes);
  *p = nullptr;
  {
    std::lock_guard<std::mutex> lk (g_pool_mu);
    auto it = g_pool.lower_bound (rb);
    if (it != g_pool.end () && it->first <= 2 * rb) {
      CachedBlock b = it->second;
      g_pool.erase (it);
      g_pool_bytes -= b.bytes;
      cudaEventSynchronize (b.ev);
      cudaEventDestroy (b.ev);
      g_live[b.p] = b.bytes;
      *p = b.p;
    }
  }
  cudaError_t e = cudaSuccess;
  if (*p == nullptr) {
    e = cudaMalloc (p, rb);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError ();
      {
        std::lock_guard<std::mutex> lk (g_pool_mu);
        pool_release_all ();
      }
      e = cudaMalloc (p, rb);
    }
    if (e == cudaSuccess) {
      std::lock_guard<std::mutex> lk (g_pool_mu);
      g_live[*p] = rb;
    }
  }
  rt_add (g_rt.alloc_s, g_rt.allocs, wall () - t0);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError ();
    return set_error (LGH_ERR_MEM, "cudaMalloc(%zu): %s", bytes,
                      cudaGetErrorString (e));
  }
  return 0;
}

void
dfree (void *p)
{
  if (!p) return;
  const double t0 = wall ();
  std::lock_guard<std::mutex> lk (g_pool_mu);
  auto it = g_live.find (p);
  size_t bytes = 0;
  if (it != g_live.end ()) {
    bytes = it->second;
    g_live.erase (it);
  }
  if (g_pool_cap == 0) {
    size_t fb = 0, tb = 0;
    if (cudaMemGetInfo (&fb, &tb) == cudaSuccess) g_pool_cap = tb / 3;
    else cudaGetLastError ();
  }
  cudaEvent_t ev = nullptr;
  if (bytes == 0 || g_pool_bytes + bytes > g_pool_cap
      || cudaEventCreateWithFlags (&ev, cudaEventDisableTiming) != cudaSuccess
      || cudaEventRecord (ev, stream ()) != cudaSuccess) {
    if (ev) cudaEventDestroy (ev);
    cudaGetLastError ();
    cudaFree (p);
  } else {
    g_pool.insert ({ bytes, CachedBlock{ p, bytes, ev } });
    g_pool_bytes += bytes;
  }
  rt_add (g_rt.free_s, g_rt.frees, wall () - t0);
}

/* ---- CSR helpers --------------------------------------------------------- */

__global__ void
k_csr_diag (int64_t n, const int64_t *rowptr, const int32_t *col,
            const double *vals, double *dinv, float *dinv32, float *vals32,
            int *maxnnz)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x) {
    double d = 0.;
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; k++) {
      if (col[k] == i) d += vals[k];
      vals32[k] = (float) vals[k];
    }
    const double di = (d != 0.) ? 1. / d : 0.;
    dinv[i] = di;
    dinv32[i] = (float) di;
    atomicMax (maxnnz, (int) (rowptr[i + 1] - rowptr[i]));
  }
}

__global__ void
k_csr_vd (int64_t n, const int64_t *rowptr, const int32_t *col,
          const double *vals, const double *dinv, double *vd, float *vd32)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; k++) {
      const double v = vals[k] * dinv[col[k]];
      vd[k] = v;
      vd32[k] = (float) v;
    }
}

__global__ void
k_check_csr (int64_t n, int64_t ncols, const int64_t *rowptr, const int32_t *col,
             int *bad)
{
  /* bad[0]: malformed row pointers (1) or a column out of range (2);
   * bad[1]: the bandwidth max |j - i| (clamped to INT_MAX) */
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x) {
    if (rowptr[i + 1] < rowptr[i]) { atomicExch (bad, 1); continue; }
    int64_t bw = 0;
    for (int64_t k = rowptr[i]; k < rowptr[i + 1]; k++) {
      if (col[k] < 0 || col[k] >= ncols) atomicExch (bad, 2);
      const int64_t d = col[k] > i ? col[k] - i : i - col[k];
      if (d > bw) bw = d;
    }
    if (bw > 0) atomicMax (bad + 1, (int) (bw < 0x7fffffff ? bw : 0x7fffffff));
  }
}

int
csr_finish (Csr &A)
{
  cudaStream_t s = stream ();
  LGH_TRY (dalloc ((void **) &A.vals32, (size_t) A.nnz * sizeof (float) + 16));
  LGH_TRY (dalloc ((void **) &A.dinv, (size_t) A.n * sizeof (double) + 16));
  LGH_TRY (dalloc ((void **) &A.dinv32, (size_t) A.n * sizeof (float) + 16));
  DBuf<int> flags;
  LGH_TRY (flags.alloc (2));
  LGH_CUDA (cudaMemsetAsync (flags.p, 0, 2 * sizeof (int), s));
  const int grid = (int) std::min<int64_t> ((A.n + 255) / 256 + 1, num_sms () * 16);
  k_check_csr<<<grid, 256, 0, s>>> (A.n, A.ncols > 0 ? A.ncols : A.n,
                                    A.rowptr, A.colidx, flags.p);
  LGH_LAUNCH_CHECK ();
  int h[2];
  LGH_CUDA (cudaMemcpyAsync (h, flags.p, 2 * sizeof (int), cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  LGH_CHECK (h[0] == 0, LGH_ERR_ARG_WRONG, "csr: malformed row pointers or column index out of range");
  A.bandwidth = h[1];
  LGH_CUDA (cudaMemsetAsync (flags.p, 0, sizeof (int), s));
  k_csr_diag<<<grid, 256, 0, s>>> (A.n, A.rowptr, A.colidx, A.vals, A.dinv,
                                   A.dinv32, A.vals32, flags.p);
  LGH_LAUNCH_CHECK ();
  LGH_CUDA (cudaMemcpyAsync (h, flags.p, sizeof (int), cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  A.max_row_nnz = h[0];
  if (A.ncols == 0 || A.ncols == A.n) {
    LGH_TRY (dalloc ((void **) &A.vd, (size_t) A.nnz * sizeof (double) + 16));
    LGH_TRY (dalloc ((void **) &A.vd32, (size_t) A.nnz * sizeof (float) + 16));
    k_csr_vd<<<grid, 256, 0, s>>> (A.n, A.rowptr, A.colidx, A.vals, A.dinv,
                                   A.vd, A.vd32);
    LGH_LAUNCH_CHECK ();
    LGH_CUDA (cudaStreamSynchronize (s));
  }
  return 0;
}

void
csr_free (Csr &A)
{
  dfree (A.rowptr);
  dfree (A.colidx);
  dfree (A.vals);
  dfree (A.vals32);
  dfree (A.dinv);
  dfree (A.dinv32);
  dfree (A.vd);
  dfree (A.vd32);
  A = Csr ();
}

} /* namespace lgh */

using namespace lgh;

/* ======================================================================== */
/* C ABI                                                                    */

extern "C" {

const char *
lgh_last_error (void)
{
  return g_err.c_str ();
}

int
lgh_runtime_counters (double *out)
{
  LGH_CHECK (out, LGH_ERR_ARG_NULL, "lgh_runtime_counters: NULL");
  std::lock_guard<std::mutex> lk (g_rt_mu);
  out[0] = (double) g_rt.allocs;
  out[1] = g_rt.alloc_s;
  out[2] = (double) g_rt.frees;
  out[3] = g_rt.free_s;
  out[4] = (double) __atomic_load_n (&lgh::g_launches, __ATOMIC_RELAXED);
  return 0;
}

long
lgh_launch_count (void)
{
  return __atomic_load_n (&lgh::g_launches, __ATOMIC_RELAXED);
}

int
lgh_mat_create_csr (int64_t n, const int64_t *rowptr, const int32_t *colidx,
                    const double *vals, int where, lgh_Mat *out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (out && rowptr && (n == 0 || (colidx && vals)), LGH_ERR_ARG_NULL,
             "lgh_mat_create_csr: NULL argument");
  LGH_CHECK (n > 0 && n < (int64_t) INT32_MAX, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_mat_create_csr: n=%lld out of range", (long long) n);
  cudaStream_t s = stream ();
  const cudaMemcpyKind kind = (where == LGH_MEM_DEVICE) ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyHostToDevice;
  int64_t nnz = 0;
  if (where == LGH_MEM_DEVICE)
    LGH_CUDA (cudaMemcpy (&nnz, rowptr + n, sizeof (int64_t), cudaMemcpyDeviceToHost));
  else
    nnz = rowptr[n];
  LGH_CHECK (nnz >= 0, LGH_ERR_ARG_WRONG, "lgh_mat_create_csr: nnz < 0");
  lgh_mat_s *A = new lgh_mat_s ();
  A->refs = 1;
  A->kind = 0;
  A->csr.n = n;
  A->csr.nnz = nnz;
  int rc = dalloc ((void **) &A->csr.rowptr, (size_t) (n + 1) * sizeof (int64_t));
  if (!rc) rc = dalloc ((void **) &A->csr.colidx, (size_t) nnz * sizeof (int32_t) + 16);
  if (!rc) rc = dalloc ((void **) &A->csr.vals, (size_t) nnz * sizeof (double) + 16);
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync (A->csr.rowptr, rowptr, (size_t) (n + 1) * sizeof (int64_t), kind, s);
    if (e == cudaSuccess && nnz)
      e = cudaMemcpyAsync (A->csr.colidx, colidx, (size_t) nnz * sizeof (int32_t), kind, s);
    if (e == cudaSuccess && nnz)
      e = cudaMemcpyAsync (A->csr.vals, vals, (size_t) nnz * sizeof (double), kind, s);
    if (e != cudaSuccess) rc = set_error (LGH_ERR_GPU, "lgh_mat_create_csr: copy: %s", cudaGetErrorString (e));
  }
  if (!rc) rc = csr_finish (A->csr);
  if (rc) {
    csr_free (A->csr);
    delete A;
    return rc;
  }
  *out = A;
  return 0;
}

int
lgh_mat_create_dense (int64_t n, const double *a, int64_t lda, int where,
                      lgh_Mat *out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (a && out, LGH_ERR_ARG_NULL, "lgh_mat_create_dense: NULL argument");
  LGH_CHECK (n > 0 && lda >= n && n * n < (int64_t) INT32_MAX, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_mat_create_dense: bad size");
  std::vector<double> h ((size_t) n * lda);
  if (where == LGH_MEM_DEVICE)
    LGH_CUDA (cudaMemcpy (h.data (), a, h.size () * sizeof (double), cudaMemcpyDeviceToHost));
  else
    memcpy (h.data (), a, h.size () * sizeof (double));
  std::vector<int64_t> rp (n + 1);
  std::vector<int32_t> ci ((size_t) n * n);
  std::vector<double> v ((size_t) n * n);
  for (int64_t i = 0; i <= n; i++) rp[i] = i * n;
  for (int64_t i = 0; i < n; i++)
    for (int64_t j = 0; j < n; j++) {
      ci[i * n + j] = (int32_t) j;
      v[i * n + j] = h[i + j * lda];
    }
  return lgh_mat_create_csr (n, rp.data (), ci.data (), v.data (), LGH_MEM_HOST, out);
}

int
lgh_mat_get_info (lgh_Mat A, int64_t *n, int64_t *nnz)
{
  LGH_CHECK (A, LGH_ERR_ARG_NULL, "lgh_mat_get_info: NULL");
  if (A->kind == 0) {
    if (n) *n = A->csr.n;
    if (nnz) *nnz = A->csr.nnz;
  } else {
    if (n) *n = A->nrows;
    if (nnz) *nnz = A->nrows * A->ncols;
  }
  return 0;
}

int
lgh_mat_mult (lgh_Mat A, lgh_Vec x, lgh_Vec y)
{
  LGH_CHECK (A && x && y, LGH_ERR_ARG_NULL, "lgh_mat_mult: NULL");
  LGH_CHECK (A->kind == 0, LGH_ERR_SUP, "lgh_mat_mult: not a CSR operator");
  LGH_CHECK (x->n == A->csr.n && y->n == A->csr.n, LGH_ERR_ARG_SIZ, "lgh_mat_mult: size");
  LGH_CHECK (x->d != y->d, LGH_ERR_ARG_WRONG, "lgh_mat_mult: in/out alias");
  LGH_TRY (lgh::mat_mult_vec (A, x->d, y->d));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  return 0;
}

int
lgh_mat_dense_get_array (lgh_Mat X, double **data, int64_t *nrows, int *ncols,
                         int64_t *ld)
{
  LGH_CHECK (X && X->kind == 1, LGH_ERR_ARG_WRONG, "lgh_mat_dense_get_array: not a dense block");
  if (data) *data = X->data;
  if (nrows) *nrows = X->nrows;
  if (ncols) *ncols = X->ncols;
  if (ld) *ld = X->ld;
  return 0;
}

int
lgh_mat_destroy (lgh_Mat *A)
{
  if (!A || !*A) return 0;
  lgh::mat_release (*A);
  *A = nullptr;
  return 0;
}

int
lgh_vec_create (int64_t n, lgh_Vec *v)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (v, LGH_ERR_ARG_NULL, "lgh_vec_create: NULL");
  LGH_CHECK (n > 0, LGH_ERR_ARG_OUTOFRANGE, "lgh_vec_create: n <= 0");
  lgh_vec_s *x = new lgh_vec_s ();
  x->n = n;
  x->owns = 1;
  int rc = dalloc ((void **) &x->d, (size_t) n * sizeof (double));
  if (rc) { delete x; return rc; }
  cudaMemsetAsync (x->d, 0, (size_t) n * sizeof (double), stream ());
  *v = x;
  return 0;
}

int
lgh_vec_create_with_array (int64_t n, double *device_array, lgh_Vec *v)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (v && device_array, LGH_ERR_ARG_NULL, "lgh_vec_create_with_array: NULL");
  lgh_vec_s *x = new lgh_vec_s ();
  x->n = n;
  x->owns = 0;
  x->d = device_array;
  *v = x;
  return 0;
}

int
lgh_vec_get_array (lgh_Vec v, double **device_array, int64_t *n)
{
  LGH_CHECK (v, LGH_ERR_ARG_NULL, "lgh_vec_get_array: NULL");
  if (device_array) *device_array = v->d;
  if (n) *n = v->n;
  return 0;
}

int
lgh_vec_set_host (lgh_Vec v, const double *host)
{
  LGH_CHECK (v && host, LGH_ERR_ARG_NULL, "lgh_vec_set_host: NULL");
  LGH_CUDA (cudaMemcpy (v->d, host, (size_t) v->n * sizeof (double), cudaMemcpyHostToDevice));
  return 0;
}

int
lgh_vec_get_host (lgh_Vec v, double *host)
{
  LGH_CHECK (v && host, LGH_ERR_ARG_NULL, "lgh_vec_get_host: NULL");
  LGH_CUDA (cudaMemcpy (host, v->d, (size_t) v->n * sizeof (double), cudaMemcpyDeviceToHost));
  return 0;
}

int
lgh_vec_destroy (lgh_Vec *v)
{
  if (!v || !*v) return 0;
  if ((*v)->owns) dfree ((*v)->d);
  delete *v;
  *v = nullptr;
  return 0;
}

} /* extern "C" */

/* ======================================================================== */
/* prior                                                                    */

namespace lgh
{

void
mat_release (lgh_Mat A)
{
  if (!A || --A->refs > 0) return;
  if (A->kind == 0) csr_free (A->csr);
  strip_free (A->strips);
  rows_plan_free (A->rows);
  delete A;
}

int
mat_prepare_block (lgh_Mat A, int w)
{
  if (w >= 8 && !A->strips_built) {
    LGH_TRY (strip_build (A->csr, A->strip_R, A->strips));
    A->strips_built = 1;
  }
  return 0;
}

template <typename T>
int
mat_mult_block (lgh_Mat A, const T *X, int ldx, T *Y, int ldy, int w,
                cudaStream_t s)
{
  if (A->rows) return rows_mult_block<T> (A, X, ldx, Y, ldy, w, s);
  if (w >= 8) {
    LGH_TRY (mat_prepare_block (A, w));
    return launch_strip_spmm<T> (A->strips, X, ldx, Y, ldy, w, s);
  }
  return launch_spmm<T> (A->csr, X, ldx, Y, ldy, w, s);
}

template int mat_mult_block<double> (lgh_Mat, const double *, int, double *,
                                     int, int, cudaStream_t);
template int mat_mult_block<float> (lgh_Mat, const float *, int, float *, int,
                                    int, cudaStream_t);

int
mat_mult_vec (lgh_Mat A, const double *x, double *y)
{
  if (A->rows) return rows_mult_block<double> (A, x, 1, y, 1, 1, stream ());
  return launch_spmm<double> (A->csr, x, 1, y, 1, 1, stream ());
}

/* w = Z^{-1}-type solves and Z applies through the prior, device vectors */
int
prior_applyZ (lgh_prior_t *p, const double *x, double *y)
{
  if (p->is_mat) return mat_mult_vec (p->Z, x, y);
  lgh_vec_s vx, vy;
  vx.d = (double *) x; vx.n = p->n; vx.owns = 0;
  vy.d = y; vy.n = p->n; vy.owns = 0;
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  p->cb.applyZ (&vx, &vy, p->cb.ctx);
  LGH_CUDA (cudaDeviceSynchronize ());
  return 0;
}

static int
prior_zcfg (lgh_prior_t *p, ZsolveCfg &cfg)
{
  cfg = p->zcfg;
  return 0;
}

/* y = Z^{-1} (s_in .* x) .* s_out for a single vector (the KSP path of the
 * reference, prior.h:73-75: single vectors always run per-column CG) */
int
prior_solve_vec (lgh_prior_t *p, const double *x, const double *s_in,
                 double *y, const double *s_out)
{
  cudaStream_t s = stream ();
  if (p->rows)
    return rows_zsolve<double> (p, 1, x, 1, s_in, y, 1, s_out, p->zcfg.rtol);
  if (p->is_mat) {
    ZsolveCfg cfg;
    prior_zcfg (p, cfg);
    cfg.mode = 0;
    LGH_TRY (p->wsv.alloc (p->n, 4, 0));
    return zsolve_block<double> (p->Z->csr, cfg, p->mg, p->wsv, p->n, 1, x, 1,
                                 s_in, y, 1, s_out, &p->stats, 0, s);
  }
  /* callbacks: scale into scratch, call, scale */
  LGH_TRY (p->tmp1.alloc (p->n));
  LGH_TRY (p->tmp2.alloc (p->n));
  LGH_TRY (launch_vec_scale (p->n, x, s_in, 1.0, p->tmp1.p, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  lgh_vec_s vx, vy;
  vx.d = p->tmp1.p; vx.n = p->n; vx.owns = 0;
  vy.d = p->tmp2.p; vy.n = p->n; vy.owns = 0;
  p->cb.solveZ (&vx, &vy, p->cb.ctx);
  LGH_CUDA (cudaDeviceSynchronize ());
  return launch_vec_scale (p->n, p->tmp2.p, s_out, 1.0, y, s);
}

/* blocked solve on row-major blocks (lgh_prior_solve_block,
 * glr_common_impl.h:205-234): Mat path -> device blocked solver;
 * callbacks -> the user's blocked callback on a column-major copy, or a
 * loop over the vector callback. */
template <typename T>
int
prior_solve_rows (lgh_prior_t *p, int w, const T *X, int ldx,
                  const double *s_in, T *Y, int ldy, const double *s_out,
                  double rtol_override)
{
  cudaStream_t s = stream ();
  if (w == 0) return 0;
  if (p->rows)
    return rows_zsolve<T> (p, w, X, ldx, s_in, Y, ldy, s_out,
                           rtol_override > 0. ? rtol_override : p->zcfg.rtol);
  if (p->is_mat) {
    ZsolveCfg cfg;
    prior_zcfg (p, cfg);
    if (rtol_override > 0.) cfg.rtol = rtol_override;
    if (std::is_same<T, float>::value && p->mg != nullptr && cfg.mode <= 1) {
      /* FP32 blocks (mixed form): FP64 PCG iterates, FP32 V-cycle, FP32 in
       * and out -- FP32 Krylov vectors would stop at eps_32 kappa(Z) */
      const int64_t n = p->n;
      const int ld = round_ld (w);
      LGH_TRY (p->mix_in.alloc ((size_t) n * ld));
      LGH_TRY (launch_f32_to_f64 (n, w, (const float *) X, ldx, p->mix_in.p, ld, s));
      LGH_TRY (prior_solve_pc32 (p, w, p->mix_in.p, ld, s_in, p->mix_in.p, ld,
                                 s_out, rtol_override));
      return launch_f64_to_f32 (n, w, p->mix_in.p, ld, (float *) Y, ldy, s);
    }
    int cap = std::min (w, std::is_same<T, double>::value ? 512 : 1024);
    ZWork &ws = std::is_same<T, double>::value ? p->ws64 : p->ws32;
    LGH_TRY (ws.alloc (p->n, cap, std::is_same<T, float>::value));
    return zsolve_block<T> (p->Z->csr, cfg, p->mg, ws, p->n, w, X, ldx, s_in,
                            Y, ldy, s_out, &p->stats, 0, s);
  }
  if constexpr (std::is_same<T, float>::value) {
    return set_error (LGH_ERR_SUP, "callback priors run in FP64 only");
  } else {
    const int64_t n = p->n;
    DBuf<double> cx, cy;
    LGH_TRY (cx.alloc ((size_t) n * w));
    LGH_TRY (cy.alloc ((size_t) n * w));
    LGH_TRY (launch_rowmajor_to_colmajor (n, w, X, ldx, cx.p, n, s_in, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    if (p->cb.solveZ_blocked) {
      lgh_mat_s mx, my;
      mx.kind = my.kind = 1;
      mx.refs = my.refs = 1;
      mx.data = cx.p; my.data = cy.p;
      mx.nrows = my.nrows = n;
      mx.ncols = my.ncols = w;
      mx.ld = my.ld = n;
      p->cb.solveZ_blocked (&mx, &my, p->cb.ctx);
    } else {
      for (int j = 0; j < w; j++) {
        lgh_vec_s vx, vy;
        vx.d = cx.p + (size_t) j * n; vx.n = n; vx.owns = 0;
        vy.d = cy.p + (size_t) j * n; vy.n = n; vy.owns = 0;
        p->cb.solveZ (&vx, &vy, p->cb.ctx);
      }
    }
    LGH_CUDA (cudaDeviceSynchronize ());
    return launch_colmajor_to_rowmajor (n, w, cy.p, n, Y, ldy, s_out, s);
  }
}

int
resident_ctas (const void *fn, int threads, int smem)
{
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> cache;
  std::lock_guard<std::mutex> lk (mu);
  const auto key = std::make_pair (fn, smem * 4096 + threads);
  auto it = cache.find (key);
  if (it != cache.end ()) return it->second;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor (&per_sm, fn, threads,
                                                     (size_t) smem)
      != cudaSuccess) {
    cudaGetLastError ();
    per_sm = 0;
  }
  const int r = per_sm > 0 ? per_sm * num_sms () : 0;
  cache[key] = r;
  return r;
}

/* FP64 block solve to the prior's tolerance with an FP32 V-cycle inside
 * FP64 PCG (the mixed form's Z-solves; Jacobi or callback priors solve in
 * FP64).  X and Y may be the same block. */
int
prior_solve_pc32 (lgh_prior_t *p, int w, const double *X, int ldx,
                  const double *s_in, double *Y, int ldy, const double *s_out,
                  double rtol_override)
{
  if (w == 0) return 0;
  if (p->rows || !p->is_mat || p->mg == nullptr || p->zcfg.mode > 1)
    return prior_solve_rows<double> (p, w, X, ldx, s_in, Y, ldy, s_out,
                                     rtol_override);
  ZsolveCfg cfg;
  prior_zcfg (p, cfg);
  if (rtol_override > 0.) cfg.rtol = rtol_override;
  cfg.pc32 = 1;
  LGH_TRY (p->ws64.alloc (p->n, std::min (w, 512), 0));
  p->pc32_calls++;
  return zsolve_block<double> (p->Z->csr, cfg, p->mg, p->ws64, p->n, w, X, ldx,
                               s_in, Y, ldy, s_out, &p->stats, 0, stream ());
}

template int prior_solve_rows<double> (lgh_prior_t *, int, const double *, int,
                                       const double *, double *, int,
                                       const double *, double);
template int prior_solve_rows<float> (lgh_prior_t *, int, const float *, int,
                                      const double *, float *, int,
                                      const double *, double);

void
prior_ref (lgh_prior_t *p)
{
  p->refs++;
}

} /* namespace lgh */

__global__ void
k_mass_init (int64_t n, const double *mass, double *m, double *ms, double *mis)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x) {
    const double v = mass[i];
    m[i] = v;
    ms[i] = sqrt (fabs (v));
    mis[i] = 1. / ms[i];
  }
}

static int
prior_init_common (lgh_Vec mass, lgh_prior_t **out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (mass && out, LGH_ERR_ARG_NULL, "prior: NULL argument");
  lgh_prior_t *p = new lgh_prior_t ();
  p->refs = 1;
  p->n = mass->n;
  int rc = p->mass.alloc (p->n);
  if (!rc) rc = p->msqrt.alloc (p->n);
  if (!rc) rc = p->minvsqrt.alloc (p->n);
  if (rc) { delete p; return rc; }
  k_mass_init<<<std::max (1, std::min (num_sms () * 8, (int) ((p->n + 255) / 256))),
                256, 0, stream ()>>> (p->n, mass->d, p->mass.p, p->msqrt.p,
                                      p->minvsqrt.p);
  cudaError_t e = cudaStreamSynchronize (stream ());
  if (e != cudaSuccess) {
    delete p;
    return set_error (LGH_ERR_GPU, "prior: %s", cudaGetErrorString (e));
  }
  *out = p;
  return 0;
}

extern "C" {

lgh_prior_mat_opts_t
lgh_prior_mat_opts_default (void)
{
  /* glr_common_impl.h:99-112 */
  lgh_prior_mat_opts_t o;
  o.ksp_rtol = 1e-12;
  o.blocked_mode = 0;
  o.tile = 64;
  o.cheb_rtol = 1e-10;
  o.smax_krylov = 1;
  o.smoother_top = 1.1;
  o.nu_force = 0;
  o.verbose = 0;
  return o;
}

int
lgh_prior_create_callbacks (lgh_Vec mass, const lgh_prior_callbacks_t *cb,
                            lgh_prior_t **prior)
{
  /* glr_common_impl.h:134-146 */
  LGH_CHECK (cb != NULL && cb->applyZ != NULL && cb->solveZ != NULL,
             LGH_ERR_ARG_NULL,
             "lgh_prior_create_callbacks: applyZ and solveZ are required");
  LGH_TRY (prior_init_common (mass, prior));
  (*prior)->cb = *cb;
  (*prior)->is_mat = 0;
  return 0;
}

int
lgh_prior_create_mat (lgh_Mat Z, lgh_Vec mass, const lgh_prior_mat_opts_t *opts,
                      lgh_prior_t **prior)
{
  /* the preconditioner of the Mat path: aggregation multigrid (the
   * reference's PCGAMG) unless LGH_PRIOR_PC_TYPE=jacobi, the counterpart
   * of its "-lgh_prior_pc_type" option (zsolve_impl.h:816-817) */
  int pc = LGH_PC_AMG;
  const char *env = getenv ("LGH_PRIOR_PC_TYPE");
  if (env && (strcmp (env, "jacobi") == 0 || strcmp (env, "JACOBI") == 0))
    pc = LGH_PC_JACOBI;
  return lgh_prior_create_mat_pc (Z, mass, opts, pc, prior);
}

int
lgh_prior_create_mat_pc (lgh_Mat Z, lgh_Vec mass,
                         const lgh_prior_mat_opts_t *opts, int pc_type,
                         lgh_prior_t **prior)
{
  LGH_CHECK (Z && Z->kind == 0, LGH_ERR_ARG_WRONG, "lgh_prior_create_mat: Z must be a CSR Mat");
  LGH_CHECK (mass && mass->n == Z->csr.n, LGH_ERR_ARG_SIZ, "lgh_prior_create_mat: mass size");
  lgh_prior_mat_opts_t o = opts ? *opts : lgh_prior_mat_opts_default ();
  LGH_CHECK (o.blocked_mode >= 0 && o.blocked_mode <= 3, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_prior_create_mat: blocked_mode %d", o.blocked_mode);
  LGH_CHECK (pc_type == LGH_PC_AMG || pc_type == LGH_PC_JACOBI,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_prior_create_mat: pc type %d", pc_type);
  LGH_CHECK (o.blocked_mode != 3 || pc_type == LGH_PC_AMG, LGH_ERR_ARG_WRONG,
             "lgh_prior_create_mat: blocked_mode 3 needs the multigrid "
             "preconditioner");
  LGH_CHECK (!Z->rows || o.blocked_mode <= 1, LGH_ERR_SUP,
             "lgh_prior_create_mat: a row-sharded Z solves with PCG "
             "(blocked_mode 0 or 1)");
  lgh_prior_t *p;
  LGH_TRY (prior_init_common (mass, &p));
  p->is_mat = 1;
  p->Z = Z;
  Z->refs++;
  p->mopts = o;
  p->pc_type = pc_type;
  if (Z->rows) {
    /* the rank-local block-Jacobi preconditioner on the diagonal block */
    p->rows = new RowsPrior ();
    int rc = rows_prior_setup (p);
    if (rc) { lgh_prior_destroy (p); return rc; }
    if (o.verbose && p->mg)
      printf ("lgh_prior: rank %d multigrid %d levels (coarse %d) setup "
              "%.3f s\n", Z->rows->comm.rank, (int) p->mg->lev.size (),
              p->mg->n0, p->mg->setup_s);
  } else if (pc_type == LGH_PC_AMG) {
    const int nu = o.nu_force > 0 ? o.nu_force : 2;
    int rc = mg_build (Z->csr, o.tile, o.smoother_top, nu, &p->mg);
    if (rc) { lgh_prior_destroy (p); return rc; }
    if (o.verbose)
      printf ("lgh_prior: multigrid %d levels (coarse %d) setup %.3f s\n",
              (int) p->mg->lev.size (), p->mg->n0, p->mg->setup_s);
  }
  p->zcfg.mode = o.blocked_mode;
  p->zcfg.rtol = o.ksp_rtol;
  p->zcfg.maxit = 10000;
  p->zcfg.tile = o.tile;
  p->zcfg.cheb_rtol = o.cheb_rtol;
  if (o.blocked_mode >= 2) {
    /* spectral bounds from a CG-Lanczos solve on the deterministic probe
     * randn_at(0xB0BD5, i, 0), rtol 1e-12, 200 its; widened by 0.9 / 1.1
     * (zsolve_impl.h:737-764) */
    const int64_t n = p->n;
    cudaStream_t s = stream ();
    DBuf<double> rhs, y;
    int rc = rhs.alloc (n);
    if (!rc) rc = y.alloc (n);
    if (!rc) rc = launch_sketch (0xB0BD5ULL, n, 0, 1, rhs.p, 1, s);
    ZsolveCfg bc = p->zcfg;
    bc.mode = 0;
    bc.rtol = 1e-12;
    bc.maxit = 200;
    bc.check_every = 1000000;
    if (!rc) rc = p->wsv.alloc (n, 4, 0);
    ZsolveStats st;
    if (!rc) rc = zsolve_block<double> (Z->csr, bc, p->mg, p->wsv, n, 1, rhs.p,
                                        1, nullptr, y.p, 1, nullptr, &st, 1, s);
    int its = (int) st.col_iters;
    if (!rc && its < 1) rc = set_error (LGH_ERR_NOT_CONVERGED, "prior: bound probe ran 0 iterations");
    std::vector<double> hist (2 * (size_t) std::max (its, 1));
    if (!rc) {
      cudaError_t e = cudaMemcpy (hist.data (), p->wsv.hist.p,
                                  2 * its * sizeof (double), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = set_error (LGH_ERR_GPU, "prior: %s", cudaGetErrorString (e));
    }
    double emin = 0., emax = 0.;
    if (!rc) {
      std::vector<double> al (its), be (its);
      for (int k = 0; k < its; k++) { al[k] = hist[2 * k]; be[k] = hist[2 * k + 1]; }
      rc = device_tridiag_extremes (its, al.data (), be.data (), &emin, &emax);
    }
    if (rc) { lgh_prior_destroy (p); return rc; }
    p->emin = emin;
    p->emax = emax;
    p->bound_its = its;
    p->zcfg.lmin = 0.9 * emin;
    p->zcfg.lmax = 1.1 * emax;
    {
      const double kap = p->zcfg.lmax / p->zcfg.lmin;
      const double rho = (sqrt (kap) - 1.) / (sqrt (kap) + 1.);
      p->zcfg.nit = (int) ceil (log (2. / o.cheb_rtol) / log (1. / rho));
    }
    if (o.verbose)
      printf ("lgh_prior: mode %d bounds [%.3e, %.3e] (%d its) -> chebyshev nit %d\n",
              o.blocked_mode, emin, emax, its, p->zcfg.nit);
  }
  *prior = p;
  return 0;
}

int
lgh_prior_create_ksp (lgh_KSP ksp, lgh_Vec mass, const lgh_prior_mat_opts_t *opts,
                      lgh_prior_t **prior)
{
  (void) ksp; (void) mass; (void) opts; (void) prior;
  return set_error (LGH_ERR_SUP,
                    "lgh_prior_create_ksp: no PETSc KSP on this device; use "
                    "lgh_prior_create_mat or lgh_prior_create_callbacks");
}

void
lgh_prior_destroy (lgh_prior_t *prior)
{
  if (prior == NULL || --prior->refs > 0) return;
  /* the hierarchy borrows the finest operator's arrays: it goes first */
  if (prior->mg) mg_destroy (prior->mg);
  rows_prior_free (prior->rows);
  if (prior->Z) mat_release (prior->Z);
  delete prior;
}

int
lgh_prior_apply (lgh_prior_t *p, lgh_Vec x, lgh_Vec y)
{
  /* y = R x = Z M^{-1} Z^T x (glr_common_impl.h:236-244) */
  LGH_CHECK (p && x && y, LGH_ERR_ARG_NULL, "lgh_prior_apply: NULL");
  LGH_CHECK (x->n == p->n && y->n == p->n, LGH_ERR_ARG_SIZ, "lgh_prior_apply: size");
  LGH_TRY (p->tmp1.alloc (p->n));
  LGH_TRY (p->tmp2.alloc (p->n));
  LGH_TRY (prior_applyZ (p, x->d, p->tmp1.p));
  LGH_TRY (launch_vec_div (p->n, p->tmp1.p, p->mass.p, p->tmp2.p, stream ()));
  LGH_TRY (prior_applyZ (p, p->tmp2.p, y->d));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  return 0;
}

int
lgh_prior_solve (lgh_prior_t *p, lgh_Vec x, lgh_Vec y)
{
  LGH_CHECK (p && x && y, LGH_ERR_ARG_NULL, "lgh_prior_solve: NULL");
  LGH_CHECK (x->n == p->n && y->n == p->n, LGH_ERR_ARG_SIZ, "lgh_prior_solve: size");
  LGH_TRY (prior_solve_vec (p, x->d, nullptr, y->d, nullptr));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  return 0;
}

int
lgh_prior_solve_block (lgh_prior_t *p, int m, const double *X, int64_t ldx,
                       double *Y, int64_t ldy)
{
  LGH_CHECK (p && X && Y, LGH_ERR_ARG_NULL, "lgh_prior_solve_block: NULL");
  LGH_CHECK (m > 0 && ldx >= p->n && ldy >= p->n, LGH_ERR_ARG_SIZ, "lgh_prior_solve_block: size");
  cudaStream_t s = stream ();
  const int ld = round_ld (m);
  DBuf<double> a, b;
  LGH_TRY (a.alloc ((size_t) p->n * ld));
  LGH_TRY (b.alloc ((size_t) p->n * ld));
  LGH_TRY (launch_colmajor_to_rowmajor (p->n, m, X, ldx, a.p, ld, nullptr, s));
  LGH_TRY (prior_solve_rows<double> (p, m, a.p, ld, nullptr, b.p, ld, nullptr));
  LGH_TRY (launch_rowmajor_to_colmajor (p->n, m, b.p, ld, Y, ldy, nullptr, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

/* Diagnostics of the prior's Z-solver (testing): out[0..7] = emin, emax,
 * lmin, lmax, nit, bound_its, mean per-column iterations, solves. */
int
lgh_prior_get_info (const lgh_prior_t *p, double *out)
{
  LGH_CHECK (p && out, LGH_ERR_ARG_NULL, "lgh_prior_get_info: NULL");
  out[0] = p->emin;
  out[1] = p->emax;
  out[2] = p->zcfg.lmin;
  out[3] = p->zcfg.lmax;
  out[4] = p->zcfg.nit;
  out[5] = p->bound_its;
  out[6] = p->stats.cols ? (double) p->stats.col_iters / p->stats.cols : 0.;
  out[7] = (double) p->stats.calls;
  out[8] = p->mg ? (double) p->mg->lev.size () : 0.;
  out[9] = p->mg ? (double) p->mg->n0 : 0.;
  out[10] = p->mg ? p->mg->setup_s : 0.;
  out[11] = p->pc_type;
  out[12] = (double) p->pc32_calls;
  out[13] = 0.;
  return 0;
}

} /* extern "C" */
