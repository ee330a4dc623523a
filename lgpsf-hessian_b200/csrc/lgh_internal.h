/* lgh_internal.h -- shared internals of the B200 GLR library.
 *
 * Layout in HBM: every tall block (sketch, Q, Y, Z-solve iterates, U) is
 * ROW-major, N rows x w columns with a leading dimension ld that is a
 * multiple of 4 (16-byte rows for float, 32-byte for double) and a 256-byte
 * aligned base, so one nonzero of a sparse operator gathers one contiguous
 * row segment with 16-byte vector loads.  The reference's column-major
 * MATDENSE layout appears only at the C-ABI boundary (Vec, batch blocks,
 * callback blocks) and is converted there.  Small dense matrices (ell x ell)
 * are column-major FP64, LAPACK style.
 */

#ifndef LGH_INTERNAL_H
#define LGH_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/lgh_b200.h"

namespace lgh
{

/* ---- errors ------------------------------------------------------------ */

int set_error (int code, const char *fmt, ...);
void clear_error ();

#define LGH_CUDA(call)                                                       \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return ::lgh::set_error (LGH_ERR_GPU, "%s:%d %s: %s", __FILE__,        \
                               __LINE__, #call, cudaGetErrorString (e_));    \
  } while (0)

#define LGH_CHECK(cond, code, ...)                                           \
  do {                                                                       \
    if (!(cond)) return ::lgh::set_error (code, __VA_ARGS__);                \
  } while (0)

#define LGH_TRY(expr)                                                        \
  do {                                                                       \
    int rc_ = (expr);                                                        \
    if (rc_) return rc_;                                                     \
  } while (0)

extern long g_launches;

/* host-side runtime counters (lgh_runtime_counters) */
struct RuntimeCounters
{
  long allocs = 0, frees = 0;
  double alloc_s = 0., free_s = 0.;
};
extern RuntimeCounters g_rt;

#define LGH_LAUNCH_CHECK()                                                   \
  do {                                                                       \
    __atomic_fetch_add (&::lgh::g_launches, 1L, __ATOMIC_RELAXED);           \
    cudaError_t e_ = cudaGetLastError ();                                    \
    if (e_ != cudaSuccess)                                                   \
      return ::lgh::set_error (LGH_ERR_GPU, "%s:%d launch: %s", __FILE__,    \
                               __LINE__, cudaGetErrorString (e_));           \
  } while (0)

/* ---- runtime ------------------------------------------------------------ */

cudaStream_t stream ();
int num_sms ();
int ensure_init ();
double wall ();

/* device allocation helpers (return LGH_ERR_MEM on failure) */
int dalloc (void **p, size_t bytes);
void dfree (void *p);
/* bytes of freed blocks the allocation cache holds: dalloc reuses them,
 * or releases them all and retries when the device is out of memory, so
 * they count as free device memory */
size_t pool_cached_bytes ();

template <typename T>
struct DBuf
{
  T *p = nullptr;
  size_t n = 0;
  DBuf () = default;
  DBuf (const DBuf &) = delete;
  DBuf &operator= (const DBuf &) = delete;
  DBuf (DBuf &&o) noexcept : p (o.p), n (o.n) { o.p = nullptr; o.n = 0; }
  DBuf &operator= (DBuf &&o) noexcept
  {
    if (this != &o) {
      release ();
      p = o.p; n = o.n;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DBuf () { release (); }
  int alloc (size_t count)
  {
    if (count <= n && p) return 0;
    release ();
    int rc = dalloc ((void **) &p, count * sizeof (T) + 256);
    if (rc) return rc;
    n = count;
    return 0;
  }
  void release ()
  {
    if (p) dfree (p);
    p = nullptr;
    n = 0;
  }
  void swap (DBuf &o)
  {
    T *tp = p; p = o.p; o.p = tp;
    size_t tn = n; n = o.n; o.n = tn;
  }
};

inline int
round_ld (int w)
{
  return (w + 3) & ~3;
}

/* ---- device CSR ----------------------------------------------------------- */

struct Csr
{
  int64_t n = 0, nnz = 0;
  int64_t ncols = 0;        /* 0: square (ncols = n) */
  int64_t *rowptr = nullptr;
  int32_t *colidx = nullptr;
  double *vals = nullptr;
  float *vals32 = nullptr;
  double *dinv = nullptr;   /* 1 / diag (Jacobi), filled on demand */
  float *dinv32 = nullptr;
  double *vd = nullptr;     /* vals[k] / diag[col[k]] (square operators):
                               the Jacobi-scaled product without a
                               dependent gather of the diagonal */
  float *vd32 = nullptr;
  int max_row_nnz = 0;
  int64_t bandwidth = 0;    /* max |j - i| over the entries */
};

/* ---- kernel launchers (k_*.cu) ------------------------------------------ */

/* sketch: Y[i*ld + j] = randn_at(seed, i0 + i, j0 + j), i < n, j < k
 * (i0: the first global row of a row slab) */
int launch_sketch (uint64_t seed, int64_t n, int64_t j0, int k, double *Y,
                   int ld, cudaStream_t s, int64_t i0 = 0);
int launch_sketch_f32 (uint64_t seed, int64_t n, int64_t j0, int k,
                       float *Y, int ld, cudaStream_t s, int64_t i0 = 0);
/* the integer xorshift state (testing) */
int launch_rng_state (uint64_t seed, int64_t n, int64_t j0, int k,
                      uint64_t *S, cudaStream_t s);

/* Y = alpha * A X  (row-major blocks of width w) */
template <typename T>
int launch_spmm (const Csr &A, const T *X, int ldx, T *Y, int ldy, int w,
                 cudaStream_t s);

/* lanes per row (2^glog) and 16-byte packs per lane (ch) of the row-group
 * kernels for a block of nvec packs; kmax > 0 (the operator's longest row)
 * lets a narrow block use half the lanes with two packs each */
void row_group_shape (int nvec, int &glog, int &ch, int kmax = 0);

/* CTAs of kernel fn (threads per CTA, dynamic shared memory) that are
 * resident on the device at once (occupancy x SMs; cached per kernel).
 * Row-group kernels walk interleaved row tiles with a stride loop, so a
 * grid of exactly this size runs in one wave: the resident CTAs sweep one
 * band of rows together (stencil neighbours hit in L2) and no tail wave
 * is left. */
int resident_ctas (const void *fn, int threads, int smem);
template <typename K>
inline int
fit_grid (K kern, int want, int threads, int smem)
{
  const int r = resident_ctas ((const void *) kern, threads, smem);
  return (r > 0 && r < want) ? r : want;
}

/* Y += A X (mode 1) or Y = B - A X (mode 2) */
template <typename T>
int launch_spmm_mode (const Csr &A, const T *X, int ldx, T *Y, int ldy, int w,
                      int mode, const T *Bm, int ldb, cudaStream_t s);

/* the last two steps of a two-step post-smoothing sequence in one pass:
 * with F1 = b1 Z D^{-1} (values fl(b1 vd_ij)) and R0 the residual,
 * r1 = R0 - F1 R0, d0 = (bp dinv) R0, X += d0, X += (b dinv) r1 + a d0 */
template <typename T>
int launch_spmm_cheb_post (const Csr &F1, const T *R0, T *X, int ld, int w,
                           const T *dinv, double a, double b, double bp,
                           cudaStream_t s);

/* the coarse correction and the whole two-step post-smoothing in one
 * pass: X += P Xc (the prolongation), then the two steps of
 * launch_spmm_cheb_post from the post residual R */
template <typename T>
int launch_post_prolong (const Csr &F1, const Csr &P, const T *R, const T *Xc,
                         T *X, int ld, int w, const T *dinv, double a,
                         double b, double bp, cudaStream_t s);

/* Y = (TO) X over count elements of two blocks with the same layout */
template <typename TI, typename TO>
int cvt_flat (int64_t count, const TI *X, TO *Y, cudaStream_t s);

/* elementwise / block helpers (k_vec.cu) */
template <typename T>
int launch_rowscale (int64_t n, int w, const double *scale, const T *X,
                     int ldx, T *Y, int ldy, cudaStream_t s);
template <typename T>
int launch_copy_block (int64_t n, int w, const T *X, int ldx, T *Y, int ldy,
                       cudaStream_t s);
int launch_colmajor_to_rowmajor (int64_t n, int w, const double *X,
                                 int64_t ldx, double *Y, int ldy,
                                 const double *scale, cudaStream_t s);
int launch_rowmajor_to_colmajor (int64_t n, int w, const double *X, int ldx,
                                 double *Y, int64_t ldy, const double *scale,
                                 cudaStream_t s);
int launch_f64_to_f32 (int64_t n, int w, const double *X, int ldx, float *Y,
                       int ldy, cudaStream_t s);
int launch_f32_to_f64 (int64_t n, int w, const float *X, int ldx, double *Y,
                       int ldy, cudaStream_t s);
int launch_zero_block (int64_t n, int ld, void *Y, size_t elem,
                       cudaStream_t s);
/* out[j] = || X[:, j] - lam[j] * U[:, j] ||_2 over all rows (FP64) */
template <typename T>
int launch_resid_norms (int64_t n, int w, const T *FU, int ldf, const T *U,
                        int ldu, const double *lam, double *out,
                        double *partials, unsigned *counter, cudaStream_t s);
/* y = x (.) scale, vectors */
int launch_vec_scale (int64_t n, const double *x, const double *scale,
                      double alpha, double *y, cudaStream_t s);
int launch_vec_axpby (int64_t n, double a, const double *x, double b,
                      const double *y, double *out, cudaStream_t s);

/* dense (k_gemm.cu): C = A^T B over n rows (split-K, FP64 accumulate),
 * C is m1 x m2 column-major with leading dim ldc; sym: 1 => C = (C + C^T)/2 */
template <typename T>
int launch_gemm_tn (int64_t n, int m1, int m2, const T *A, int lda,
                    const T *B, int ldb, double *C, int ldc, int sym,
                    double *work, size_t work_elems, cudaStream_t s);
/* Y = alpha X M + beta Y0; X n x k row-major, M k x m2 column-major FP64
 * (leading dim ldm); Y, Y0 row-major */
template <typename T>
int launch_gemm_nn (int64_t n, int k, int m2, double alpha, const T *X,
                    int ldx, const double *M, int ldm, double beta,
                    const T *Y0, int ldy0, T *Y, int ldy, cudaStream_t s);
size_t gemm_tn_work_elems (int64_t n, int m1, int m2);

/* partial-sum elements enough for every gemm_tn shape up to m1max x m2max */
size_t gemm_tn_work_max (int m1max, int m2max);
/* Y = A^{-1} B for a dense n0 x n0 column-major A^{-1} and row-major B, Y
 * (n0 x ld); columns w .. ld - 1 of Y are zeroed */
template <typename T>
int launch_dense_apply (int n0, const double *Ainv, const T *B, T *Y, int w,
                        int ld, cudaStream_t s);

/* small dense FP64 (k_small.cu), matrices column-major n x n, ld n */
/* Cholesky (lower) with the reference's single jitter retry; info[0] = 0
 * ok, 1 failed twice; info[1] = 1 if the jitter was used.  jitter_mode 0:
 * + 1e-12 tr/n (glr_common_impl.h:386-396); 1: + 1e-12 max(dmax, 1)
 * (glr_scalapack_impl.h:129-139). */
int launch_potrf (int n, double *G, double *G0, int jitter_mode, int *info,
                  cudaStream_t s);
/* Linv = L^{-1} (lower), transposed on request: out = (L^{-1})^T */
int launch_trtri_lower (int n, const double *L, double *Linv, int transpose,
                        cudaStream_t s);
/* symmetric eigensolve: A (destroyed) -> w (unordered), V (column-major) */
int launch_syev_jacobi (int n, double *A, double *V, double *w, double *A2,
                        double *V2, int *sweeps, cudaStream_t s);
/* order by |w| desc; cut = max(trunc_abs, trunc_rel*max|w|); fills
 * order[n], sel[6] = {kept, absmax, next_abs, raw_min, raw_max, nneg},
 * lam[kept] treated; C (n x kept col-major) = V[:, order[0:kept]] */
int launch_select (int n, const double *w, const double *V, double trunc_abs,
                   double trunc_rel, int treat, int *order, double *sel,
                   double *lam, double *C, cudaStream_t s);
/* symmetric tridiagonal (diag d, off e) eigen extremes through Jacobi */
int device_tridiag_extremes (int m, const double *alpha,
                             const double *beta, double *emin, double *emax);

/* ---- Z-solve (zsolve.cu) ------------------------------------------------ */

struct ZsolveCfg
{
  int mode = 0;          /* 0/1 PCG, 2 Chebyshev, 3 Chebyshev + V-cycle */
  double rtol = 1e-12;
  int maxit = 10000;
  int tile = 64;
  double cheb_rtol = 1e-10;
  double lmin = 0, lmax = 0; /* margined interval (mode 2/3) */
  int nit = 0;
  int check_every = 16;
  int pc32 = 0;          /* FP64 PCG with an FP32 V-cycle (mixed form)  */
};

struct Hierarchy; /* aggregation multigrid (mode 3) */

struct ZsolveStats
{
  long calls = 0, block_iters = 0, col_iters = 0, cols = 0;
  double seconds = 0.;
  int last_maxit_hit = 0;
};

/* Workspace for blocked solves of width <= cap. */
struct ZWork
{
  int cap = 0;
  int64_t n = 0;
  int is32 = 0;
  DBuf<char> X, R, P0, P1, Q, Zb;
  DBuf<char> R32, Z32;         /* FP32 V-cycle input / output (pc32) */
  DBuf<double> partA, partB;   /* [nblocks][ld] */
  DBuf<double> scal;           /* per-column scalars */
  DBuf<int> ival;              /* active flags / counts */
  DBuf<unsigned> counters;
  DBuf<double> hist;           /* alpha/beta history for Lanczos */
  int nblocks = 0;
  int alloc (int64_t n, int cap, int is32);
};

/* Solve Z Y = S X (row-major blocks, width w <= any); rowscale_in
 * (nullable) scales the right-hand side rows, rowscale_out the solution.
 * T selects FP64 or FP32 iterates.  Returns LGH_ERR_NOT_CONVERGED only if
 * fail_on_maxit. */
template <typename T>
int zsolve_block (const Csr &Z, const ZsolveCfg &cfg, Hierarchy *mg,
                  ZWork &ws, int64_t n, int w, const T *X, int ldx,
                  const double *rowscale_in, T *Y, int ldy,
                  const double *rowscale_out, ZsolveStats *st,
                  int record_hist, cudaStream_t s);

/* residual-norm helper used by the tests:
 * out[c] = || D^{-1}(B - Z X) ||_2 per column (FP64) */
int zsolve_residual_norms (const Csr &Z, int64_t n, int w, const double *Bm,
                           int ldb, const double *X, int ldx, double *out,
                           cudaStream_t s);

/* mode 3: build / destroy the hierarchy from Z (device), CSR on host */
int mg_build (const Csr &Z, int tile, double smoother_top, int nu,
              Hierarchy **out);
void mg_destroy (Hierarchy *h);

} /* namespace lgh */

#endif /* LGH_INTERNAL_H */
