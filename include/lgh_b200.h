/* lgh_b200.h -- C ABI of the B200 (sm_100a) GLR library.
 *
 * A drop-in for the GLR + prior path of NickAlger/lgpsf-hessian: the same
 * lgh_prior_* / lgh_glr_* names, argument order, option/report structs
 * (field for field) and error codes as the reference headers
 *   include/lgpsf_hessian/prior.h:38-110
 *   include/lgpsf_hessian/glr.h:50-169
 *   include/lgpsf_hessian/lgpsf_hessian.h:19-43 (conventions),
 * with PETSc replaced by three opaque handle types:
 *
 *   Mat  a device-resident operator: a CSR matrix (lgh_mat_create_csr /
 *        lgh_mat_create_dense) or a dense column block handed to blocked
 *        prior callbacks.  The engine only ever multiplies by B and Z
 *        (glr.h:104-108).
 *   Vec  a device vector of doubles (lgh_vec_create / _with_array).
 *   KSP  accepted by lgh_prior_create_ksp only to return LGH_ERR_SUP.
 *
 * Conventions (lgpsf_hessian.h:19-35): functions return 0 on success and a
 * nonzero PETSc-numbered code on failure; in/out Vec arguments must not
 * alias; calls on one lgh_glr_t are serialised by the caller (the object
 * owns scratch).  Every call is synchronous with respect to the host
 * unless its name ends in _async.  There is one device (the current CUDA
 * device at the first call); no MPI: the communicator is one process.
 *
 * Extensions live under new names and never change a reference signature:
 * lgh_glr_compute_ex (precision), lgh_glr_*_batch (many right-hand sides
 * and shifts), lgh_glr_get_stats, the lgh_server_* request loop, and the
 * Mat / Vec constructors.
 */

#ifndef LGH_B200_H
#define LGH_B200_H

#include <stddef.h>
#include <stdint.h>

#define LGPSF_HESSIAN_VERSION_MAJOR 0
#define LGPSF_HESSIAN_VERSION_MINOR 1
#define LGPSF_HESSIAN_VERSION_PATCH 0

/* error codes: the PETSc numbers the reference returns (lgpsf_hessian.h:
 * 27-28 and its PetscCheck sites) */
#define LGH_SUCCESS               0
#define LGH_ERR_MEM              55  /* PETSC_ERR_MEM: device allocation    */
#define LGH_ERR_SUP              56  /* PETSC_ERR_SUP                        */
#define LGH_ERR_ORDER            58  /* PETSC_ERR_ORDER: extend after correct*/
#define LGH_ERR_ARG_SIZ          60  /* PETSC_ERR_ARG_SIZ                    */
#define LGH_ERR_ARG_WRONG        62  /* PETSC_ERR_ARG_WRONG                  */
#define LGH_ERR_ARG_OUTOFRANGE   63  /* PETSC_ERR_ARG_OUTOFRANGE             */
#define LGH_ERR_ARG_WRONGSTATE   73  /* PETSC_ERR_ARG_WRONGSTATE             */
#define LGH_ERR_LIB              76  /* PETSC_ERR_LIB: factorisation failed  */
#define LGH_ERR_CONV_FAILED      82  /* PETSC_ERR_CONV_FAILED                */
#define LGH_ERR_ARG_NULL         85  /* PETSC_ERR_ARG_NULL                   */
#define LGH_ERR_NOT_CONVERGED    91  /* PETSC_ERR_NOT_CONVERGED              */
#define LGH_ERR_GPU              97  /* PETSC_ERR_GPU: CUDA runtime error    */

#ifdef __cplusplus
extern "C"
{
#endif

/* ---- PETSc-free handle types ------------------------------------------ */

typedef struct lgh_mat_s *lgh_Mat;
typedef struct lgh_vec_s *lgh_Vec;
typedef struct lgh_ksp_s *lgh_KSP;

#ifndef LGH_NO_PETSC_NAMES
typedef lgh_Mat Mat;
typedef lgh_Vec Vec;
typedef lgh_KSP KSP;
#endif

/* where a constructor's input arrays live */
#define LGH_MEM_HOST   0
#define LGH_MEM_DEVICE 1

/* Sparse symmetric operator from CSR (0-based, int64 row pointers, int32
 * column indices, sorted or not).  Arrays are copied to the device
 * (where = LGH_MEM_HOST) or device-to-device (LGH_MEM_DEVICE).  A float
 * copy of the values is kept too, for the mixed-precision path.  The
 * handle is reference counted; lgh_mat_destroy drops one reference.       */
int lgh_mat_create_csr (int64_t n, const int64_t *rowptr,
                        const int32_t *colidx, const double *vals, int where,
                        lgh_Mat *A);
/* Dense n x n operator (column-major, leading dimension lda), e.g. the
 * MPIDENSE B of the reference's tests; stored as a full CSR.             */
int lgh_mat_create_dense (int64_t n, const double *a, int64_t lda, int where,
                          lgh_Mat *A);
int lgh_mat_get_info (lgh_Mat A, int64_t *n, int64_t *nnz);
/* y = A x (MatMult). */
int lgh_mat_mult (lgh_Mat A, lgh_Vec x, lgh_Vec y);
/* Dense column block views given to blocked prior callbacks:
 * data[i + j * ld] is row i of column j (MATDENSE layout), device memory. */
int lgh_mat_dense_get_array (lgh_Mat X, double **data, int64_t *nrows,
                             int *ncols, int64_t *ld);
int lgh_mat_destroy (lgh_Mat *A);

/* Device vectors of length n.  _with_array borrows a device array.       */
int lgh_vec_create (int64_t n, lgh_Vec *v);
int lgh_vec_create_with_array (int64_t n, double *device_array, lgh_Vec *v);
int lgh_vec_get_array (lgh_Vec v, double **device_array, int64_t *n);
int lgh_vec_set_host (lgh_Vec v, const double *host);  /* H2D copy        */
int lgh_vec_get_host (lgh_Vec v, double *host);        /* D2H copy        */
int lgh_vec_destroy (lgh_Vec *v);

/* ---- prior.h ------------------------------------------------------------ */

typedef struct lgh_prior lgh_prior_t; /* opaque */

/* y = Op x on device vectors. */
typedef void (*lgh_vec_fn) (lgh_Vec x, lgh_Vec y, void *ctx);
/* Y = Op X on dense device column blocks (lgh_mat_dense_get_array). */
typedef void (*lgh_mat_fn) (lgh_Mat X, lgh_Mat Y, void *ctx);

/* prior.h:47-57 */
typedef struct lgh_prior_callbacks
{
  lgh_vec_fn applyZ;           /* required                                 */
  lgh_vec_fn applyZt;          /* NULL => Z treated as symmetric           */
  lgh_vec_fn solveZ;           /* required                                 */
  lgh_vec_fn solveZt;          /* NULL => symmetric                        */
  lgh_mat_fn solveZ_blocked;   /* optional, performance                    */
  lgh_mat_fn solveZt_blocked;  /* optional                                 */
  void      *ctx;
}
lgh_prior_callbacks_t;

int lgh_prior_create_callbacks (lgh_Vec mass_lumps,
                                const lgh_prior_callbacks_t *callbacks,
                                lgh_prior_t **prior);

/* prior.h:76-89.  On this device the Mat path solves Z with blocked,
 * per-column preconditioned CG (blocked_mode 0/1, rtol ksp_rtol, the
 * reference's per-column KSP semantics) or blocked fixed-count Chebyshev
 * (modes 2/3, cheb_rtol, bounds from a CG-Lanczos probe widened 0.9/1.1),
 * preconditioned by a block V-cycle on a smoothed-aggregation hierarchy of
 * Z (Chebyshev-Jacobi smoothers, nu = nu_force or 2, interval
 * [0.1, smoother_top] lambda_max; dense coarse solve) or by Jacobi
 * (lgh_prior_create_mat_pc).  tile caps the block width of one blocked
 * Chebyshev pass.                                                         */
typedef struct lgh_prior_mat_opts
{
  double ksp_rtol;     /* per-column solve tolerance (default 1e-12)     */
  int    blocked_mode; /* 0 (default) | 1 | 2 | 3                         */
  int    tile;         /* block width cap (default 64; 0 = no cap)       */
  double cheb_rtol;    /* Chebyshev accuracy target (default 1e-10)      */
  int    smax_krylov;  /* 1 (default): level bounds via CG-Lanczos       */
  double smoother_top; /* smoothing-interval top factor (default 1.1)    */
  int    nu_force;     /* force smoother degree (0 = default 2)          */
  int    verbose;
}
lgh_prior_mat_opts_t;

lgh_prior_mat_opts_t lgh_prior_mat_opts_default (void);

int lgh_prior_create_mat (lgh_Mat Z, lgh_Vec mass_lumps,
                          const lgh_prior_mat_opts_t *opts,
                          lgh_prior_t **prior);
/* The Mat path with an explicit preconditioner choice (lgh_prior_create_mat
 * takes it from the environment variable LGH_PRIOR_PC_TYPE, "amg" by
 * default, the counterpart of the reference's -lgh_prior_pc_type option):
 * LGH_PC_AMG is smoothed-aggregation multigrid (the role of PCGAMG; the
 * V-cycle of blocked_mode 3), LGH_PC_JACOBI the diagonal.                 */
#define LGH_PC_AMG    0
#define LGH_PC_JACOBI 1
int lgh_prior_create_mat_pc (lgh_Mat Z, lgh_Vec mass_lumps,
                             const lgh_prior_mat_opts_t *opts, int pc_type,
                             lgh_prior_t **prior);

/* Always LGH_ERR_SUP: there is no PETSc KSP on this device.              */
int lgh_prior_create_ksp (lgh_KSP ksp, lgh_Vec mass_lumps,
                          const lgh_prior_mat_opts_t *opts,
                          lgh_prior_t **prior);
void lgh_prior_destroy (lgh_prior_t *prior);
/* y = R x = Z M^{-1} Z x */
int lgh_prior_apply (lgh_prior_t *prior, lgh_Vec x, lgh_Vec y);
/* y = Z^{-1} x through the prior's single-vector solve (testing).       */
int lgh_prior_solve (lgh_prior_t *prior, lgh_Vec x, lgh_Vec y);
/* Y = Z^{-1} X on a device column block (column-major, leading dim ld),
 * through the prior's blocked solve (testing and batched callers).      */
int lgh_prior_solve_block (lgh_prior_t *prior, int m, const double *X,
                           int64_t ldx, double *Y, int64_t ldy);

/* Diagnostics of a Mat-path prior's Z-solver: out[0..13] = Lanczos emin,
 * emax, margined lmin, lmax, Chebyshev nit, probe iterations, mean
 * per-column CG iterations so far, number of solve calls, multigrid
 * levels, coarse size, multigrid setup seconds, preconditioner type,
 * number of block solves run with the FP32 V-cycle (mixed form), 0.     */
int lgh_prior_get_info (const lgh_prior_t *prior, double *out);

/* ---- glr.h --------------------------------------------------------------- */

typedef struct lgh_glr lgh_glr_t; /* opaque */

typedef enum
{
  LGH_GLR_DEFAULT    = 0,  /* the device backend, incremental extend      */
  LGH_GLR_REPLICATED = 1,  /* the device backend, extend = full rebuild   */
  LGH_GLR_SCALAPACK  = 2   /* accepted: same as DEFAULT                   */
}
lgh_glr_backend_t;

typedef enum
{
  LGH_TREAT_FLIP = 0,      /* lam <- |lam|  (default)                      */
  LGH_TREAT_RELU = 1,      /* lam <- max(lam, 0)                           */
  LGH_TREAT_NONE = 2
}
lgh_treat_t;

/* glr.h:68-86, field for field */
typedef struct lgh_glr_opts
{
  int               ell;       /* sketch width (target rank <= ell)        */
  int               q_power;   /* power-iteration passes                   */
  double            trunc_abs; /* keep treated |lam| > trunc_abs           */
  double            trunc_rel; /* ... or > trunc_rel * max|lam| (0 = off)  */
  lgh_treat_t       treat;
  unsigned long     seed;      /* hashed-sketch seed                       */
  lgh_glr_backend_t backend;
  int               nb;        /* accepted, unused (no block-cyclic T)     */
  int               panel;     /* BCGS2 panel width of the extension       */
  int               grid2d;    /* accepted, unused                         */
  int               check;     /* eigen-residual check on build            */
}
lgh_glr_opts_t;

lgh_glr_opts_t lgh_glr_opts_default (void);

/* glr.h:90-102 */
typedef struct lgh_glr_report
{
  int    kept;
  double lam_abs_max;
  double lam_raw_min, lam_raw_max;
  double next_abs;
  int    n_negative_raw;
  double resid_max;
  double t_operator, t_dense;
}
lgh_glr_report_t;

/* glr.h:104-113 */
int lgh_glr_compute (lgh_Mat B, lgh_prior_t *prior,
                     const lgh_glr_opts_t *opts, lgh_glr_t **glr,
                     lgh_glr_report_t *report);
/* glr.h:115-124 */
int lgh_glr_extend (lgh_glr_t *glr, int k_new, lgh_glr_report_t *report);
void lgh_glr_destroy (lgh_glr_t *glr);

/* full space: H(c) = B + c R (glr.h:128-158) */
int lgh_glr_solve (lgh_glr_t *glr, double c, lgh_Vec rhs, lgh_Vec x);
int lgh_glr_apply (lgh_glr_t *glr, double c, lgh_Vec v, lgh_Vec y);
int lgh_glr_sample (lgh_glr_t *glr, double c, lgh_Vec xi, lgh_Vec x);

typedef enum
{
  LGH_FACTOR_G     = 0,
  LGH_FACTOR_GT    = 1,
  LGH_FACTOR_GINV  = 2,
  LGH_FACTOR_GINVT = 3   /* == lgh_glr_sample */
}
lgh_factor_t;

int lgh_glr_factor (lgh_glr_t *glr, double c, lgh_factor_t which,
                    lgh_Vec in, lgh_Vec out);

/* prior-weighted frame (glr.h:160-169) */
double lgh_glr_logdet (lgh_glr_t *glr, double c);
int lgh_glr_pow (lgh_glr_t *glr, double c, double p, lgh_Vec in,
                 lgh_Vec out);
int lgh_glr_filter (lgh_glr_t *glr, const double *f_lam, double f_c,
                    lgh_Vec in, lgh_Vec out);
int lgh_glr_eigs (const lgh_glr_t *glr, int *nkept, const double **lam);

/* ---- extensions --------------------------------------------------------- */

/* Mixed precision: the tall blocks (sketch, F-applies, CholQR2 sweeps)
 * are FP32 with FP64 accumulation; every ell x ell operation is FP64; the
 * Z-solves keep FP64 Krylov vectors with an FP32 multigrid V-cycle as the
 * preconditioner (FP32 Krylov vectors would stop at eps_32 kappa(Z),
 * 1e-3 on a 512^2 grid), so they reach the prior's tolerance.           */
#define LGH_PREC_FP64  0   /* everything FP64 (the plain form)             */
#define LGH_PREC_MIXED 1   /* FP32 blocks and V-cycles, FP64 Krylov + core */

typedef struct lgh_exec_opts
{
  int    precision;    /* LGH_PREC_FP64 (default) | LGH_PREC_MIXED       */
  double inner_rtol;   /* mixed: Z-solve tolerance on FP32 blocks; 0
                          (default) = the prior's own                    */
  int    verbose;
  int    rank_cap;     /* keep at most rank_cap modes ("rank r,
                          oversample p" = ell r + p, rank_cap r); 0 = off */
  int    check_form;   /* the residual check (opts.check): LGH_CHECK_PROJ
                          (default) or LGH_CHECK_APPLY                    */
}
lgh_exec_opts_t;

/* Two forms of the same residual check max_j ||F u_j - lam_j u_j||
 * (glr_common_impl.h:576-600).  The reference applies F to the kept U
 * again (LGH_CHECK_APPLY: one more F-apply of kept columns, a quarter of
 * the build).  Since U = Q C and F is linear, F U = (F Q) C, and F Q is
 * the block the Rayleigh-Ritz projection has just formed: LGH_CHECK_PROJ
 * forms F U as one product of that block with C.  The two differ by the
 * Z-solve tolerance (F through inexact solves is linear to that
 * accuracy).                                                              */
#define LGH_CHECK_PROJ  0
#define LGH_CHECK_APPLY 1

lgh_exec_opts_t lgh_exec_opts_default (void);

int lgh_glr_compute_ex (lgh_Mat B, lgh_prior_t *prior,
                        const lgh_glr_opts_t *opts,
                        const lgh_exec_opts_t *exec, lgh_glr_t **glr,
                        lgh_glr_report_t *report);

/* ---- several GPUs: the sketch's columns sharded over ranks --------------
 * The reference distributes the build over MPI row slabs
 * (docs/glr-woodbury-formulas.tex:76-98).  Here every rank (one process or
 * thread per GPU) holds B, Z and the whole N x ell blocks, and applies F
 * only to its own contiguous range of sketch columns (lgh_cols_range; the
 * hashed sketch does not depend on the split).  After each F-apply one
 * all-gather rebuilds the full block on every rank; CholQR2, the
 * Rayleigh-Ritz step and the selection then run identically on all ranks,
 * so every rank ends with the same object (U, lambda), which serves
 * solves / samples / logdet locally.  The F-applies (Z-solves and B
 * products, nearly all of the build) split evenly; no halo exchange is
 * needed.  The residual check and lgh_glr_extend shard the same way.
 *
 * allgather: make recv[r * len, (r + 1) * len) equal rank r's send[0, len)
 * on every rank, for device buffers, and return 0 (nonzero: the build
 * fails with LGH_ERR_GPU).  All ranks call it the same number of times
 * with the same len.  send / recv: caller-owned device buffers of `bytes`
 * and size * bytes (bytes >= lgh_cols_exchange_bytes), or NULL for
 * buffers the library allocates; the callback receives the buffers in use.
 * The communicator must stay valid for the object's lifetime (extend).   */
typedef struct lgh_comm
{
  int    rank, size;
  void  *send, *recv;
  size_t bytes;
  int  (*allgather) (const void *send, void *recv, size_t len, void *ctx);
  void  *ctx;
}
lgh_comm_t;

/* columns [c0, c1) of a width-w block owned by `rank` of `size` (groups of
 * 4 columns, contiguous, in rank order) */
void lgh_cols_range (int w, int rank, int size, int *c0, int *c1);
/* exchange buffer bytes one rank needs for an n-row build at width ell   */
size_t lgh_cols_exchange_bytes (int64_t n, int ell, int size);
int lgh_glr_compute_cols (lgh_Mat B, lgh_prior_t *prior,
                          const lgh_glr_opts_t *opts,
                          const lgh_exec_opts_t *exec, const lgh_comm_t *comm,
                          lgh_glr_t **glr, lgh_glr_report_t *report);
/* `size` communicators for ranks run as threads of one process on one
 * device (testing the sharded path where fewer GPUs than ranks exist): the
 * all-gather meets on a host barrier (120 s limit, then LGH_ERR_GPU) and
 * copies device to device; no kernel waits for another rank.             */
int lgh_comm_local_create (int size, lgh_comm_t *comms);
void lgh_comm_local_destroy (lgh_comm_t *comms);

typedef struct lgh_glr_stats
{
  int64_t n;
  int     ell, kept, precision;
  double  t_build, t_sketch, t_zsolve, t_spmm, t_orth, t_eig, t_check;
  long    zsolve_calls, zsolve_iters;   /* block-iterations, all solves  */
  double  zsolve_mean_col_iters;        /* mean per-column iterations    */
  int64_t device_bytes;                 /* resident state of the object  */
}
lgh_glr_stats_t;

int lgh_glr_get_stats (const lgh_glr_t *glr, lgh_glr_stats_t *stats);

/* Copy U (n x kept, column-major, leading dim ld) to device memory.     */
int lgh_glr_get_U (const lgh_glr_t *glr, double *U_dev, int64_t ld);

/* Batched downstream operations on device column blocks (column-major,
 * leading dims ldr/ldx), m right-hand sides, nshift shifts c[0..nshift):
 * output block s (columns s*m .. s*m+m-1 of x) holds the result at c[s].
 * The Z-solves, which do not depend on c, run once per right-hand side;
 * with more than one shift, every shift's Woodbury combination then runs
 * in one fused tensor-core launch that writes x directly.  That tail is
 * captured as a CUDA graph on the first call of a (kind, nshift, m) shape
 * and replayed afterwards; its tile shape is picked by the library's
 * autotuner on the first call of a shape (that call times each variant
 * once; LGH_TUNE_CACHE = a file path keeps the choices across runs).    */
int lgh_glr_solve_batch (lgh_glr_t *glr, int nshift, const double *c,
                         int m, const double *rhs, int64_t ldr, double *x,
                         int64_t ldx);
int lgh_glr_sample_batch (lgh_glr_t *glr, int nshift, const double *c,
                          int m, const double *xi, int64_t ldr, double *x,
                          int64_t ldx);
int lgh_glr_logdet_batch (lgh_glr_t *glr, int nshift, const double *c,
                          double *out);
/* The batched operations' graph and tuning state (all nullable): graph
 * captures and replays of this object, the tile variant of its last
 * combination, and the shapes the autotuner has measured in the process. */
int lgh_glr_batch_info (const lgh_glr_t *glr, long *graph_captures,
                        long *graph_replays, int *tile_variant,
                        int *tuned_shapes);

/* ---- the request loop ---------------------------------------------------
 * Continuous batching of solve / sample / logdet requests on a resident GLR
 * object: a worker thread owns a block of `slots` Z-solve columns; each
 * column carries its own CG state, so requests that arrive while others run
 * join the same launches as columns free up, and a request's result does not
 * depend on what it was batched with.  Requests are admitted in arrival
 * order column by column (a request wider than the slot block runs in
 * parts); a second thread copies inputs to the device ahead of admission,
 * while the device keeps hbm_reserve of its memory free, and copies results
 * back.  A mixed-precision object (LGH_PREC_MIXED) runs its V-cycles in
 * FP32 here too.  The loop has its own streams and work
 * buffers and only reads the GLR object and its prior, so the read-only
 * operations (solve, sample, logdet and their batched forms) may be
 * called beside it; lgh_glr_extend and the destroy calls must wait until
 * lgh_server_destroy.                                                    */
typedef struct lgh_server lgh_server_t;

#define LGH_REQ_SOLVE  0   /* x = H(c)^{-1} rhs, m columns                */
#define LGH_REQ_SAMPLE 1   /* x = G^{-T} xi, m columns                    */
#define LGH_REQ_LOGDET 2   /* *out = logdet at c                          */

typedef struct lgh_server_opts
{
  int    slots;        /* Z-solve columns in flight (default 64)          */
  double hbm_reserve;  /* fraction of device memory kept free (0.05)      */
  int    verbose;
}
lgh_server_opts_t;

typedef struct lgh_server_stats
{
  long   completed, columns, ticks, pending;
  double p50_s, p99_s, max_s;   /* request latency, submit to done        */
  double columns_per_s;
  /* the loop thread's seconds in admission (staging the admitted columns),
   * in ticks (launch to the convergence mask on the host) and in harvests,
   * and the harvest count                                                  */
  double t_admit_s, t_tick_s, t_harvest_s;
  long   harvests;
  /* the copier thread's seconds moving inputs up and results down        */
  double t_up_s, t_down_s;
  /* mean fraction of the slots occupied per tick, and the mean seconds a
   * completed solve / sample request spent in each stage: submit to input
   * staged, staged to first column placed, first column placed to last
   * column harvested, last harvest to result on the host                 */
  double occupancy;
  double wait_stage_s, wait_admit_s, run_s, copy_out_s;
}
lgh_server_stats_t;

lgh_server_opts_t lgh_server_opts_default (void);
int lgh_server_create (lgh_glr_t *glr, const lgh_server_opts_t *opts,
                       lgh_server_t **server);
/* in / out: host column-major blocks (n x m, any m >= 1, leading dims
 * ldin / ldout) that stay valid until the request completes;
 * LGH_REQ_LOGDET writes one double to out.  A request that cannot get
 * device memory for its staging while nothing else holds any completes
 * with LGH_ERR_MEM (reported by lgh_server_wait); the loop carries on.    */
int lgh_server_submit (lgh_server_t *server, int kind, double c, int m,
                       const double *in, int64_t ldin, double *out,
                       int64_t ldout, int64_t *id);
/* block until request id completes (or timeout_s passes: LGH_ERR_NOT_
 * CONVERGED); latency_s (nullable) receives submit-to-done seconds.       */
int lgh_server_wait (lgh_server_t *server, int64_t id, double timeout_s,
                     double *latency_s);
int lgh_server_get_stats (lgh_server_t *server, lgh_server_stats_t *stats);
void lgh_server_destroy (lgh_server_t *server);

/* G = X^T X (w x w, column-major, ldg) of a row-major device block X
 * (n x w, ldx) without any device allocation.  No counterpart in the
 * reference: for callers that fix the device memory budget up front and
 * forbid a library to allocate.  Its split-K partial sums live in one
 * fixed 8 MiB device array inside the library, so w <= 1024 (w * w <=
 * 2^20 doubles; larger w returns LGH_ERR_ARG_OUTOFRANGE).  Every call
 * looks the array's device address up on the current device.  The call runs
 * on the legacy default stream and synchronises it before returning, so it
 * cannot run while any stream capture is active in the process.  Calls
 * share the array: calls from different host threads race on it and must
 * be serialised.                                                          */
int lgh_gram_noalloc (int64_t n, int w, const double *X, int64_t ldx,
                      double *G, int64_t ldg);

/* ---- stage 2.5: deflation correction against the true Hessian
 * (glr.h:171-270).  The GLR object approximates the misfit Hessian; the
 * correction measures the dominant modes of the whitened error operator
 *   E_w = S^- (F_true + c0 I) S^- - I,  S^- = (U lam U^T + c0 I)^{-1/2},
 *   F_true = M^{1/2} Z^{-1} H_d Z^{-T} M^{1/2},
 * with the user's true-Hessian applies, and grafts a rank-r correction into
 * (U, lam).  The corrected spectrum is SIGNED (never flipped); shift-taking
 * operations then need c > floor = max(0, -min lam'); lgh_glr_apply serves
 * the corrected low-rank action; lgh_glr_extend is refused afterwards.    */
typedef struct lgh_glr_correct_opts
{
  double        c0;        /* reference shift of the error metric (1.0)   */
  int           rank;      /* max correction rank; -1 (default) = all     */
  int           applies;   /* true-Hessian apply budget (default 30)      */
  int           n_qc;      /* probes path: trailing probes held out (0)   */
  int           q_power;   /* fresh path: extra power passes (0)          */
  double        clamp_eps; /* d clamped to >= -1 + clamp_eps (0.05)       */
  double        d_keep_min;/* drop priced modes with |d| below this (0)   */
  double        drop_tol;  /* relative basis drop tolerance (1e-12)       */
  unsigned long seed;      /* fresh-path hashed sketch seed (424242)      */
  int           verbose;
}
lgh_glr_correct_opts_t;

lgh_glr_correct_opts_t lgh_glr_correct_opts_default (void);

typedef struct lgh_glr_correct_report
{
  int    kept;             /* correction modes grafted                    */
  int    basis;            /* error-basis dimension available             */
  int    clamped;          /* Rayleigh values clamped at -1 + clamp_eps   */
  int    hd_applies;       /* true-Hessian applies spent                  */
  double d_min, d_max;     /* correction eigenvalues, post-clamp          */
  double floor;            /* shift validity: ops need c > floor          */
  double qc_before, qc_after;  /* whitened energy ratio on held-out
                                  probes (n_qc > 0); -1 when unavailable  */
  double t_operator, t_dense;
}
lgh_glr_correct_report_t;

/* y = H_d x on HOST arrays of the N dofs (the reference's local arrays on
 * one rank); the library copies each column to and from the device.     */
#ifndef LGH_HESSIAN_FN_DEFINED
#define LGH_HESSIAN_FN_DEFINED
typedef void (*lgh_hessian_fn) (const double *in_local, double *out_local,
                                void *ctx);
#endif

/* Value-pass correction from k probe pairs (host, column-major: V[j*N + i]
 * entry i of probe j, HV the true-Hessian responses); the apply budget
 * prices the top error-basis directions exactly.                         */
int lgh_glr_correct_probes (lgh_glr_t *glr, int k, const double *V,
                            const double *HV, lgh_hessian_fn hessian_apply,
                            void *ctx, const lgh_glr_correct_opts_t *opts,
                            lgh_glr_correct_report_t *report);
/* Fresh randomized correction: a hashed Gaussian sketch of E_w.          */
int lgh_glr_correct (lgh_glr_t *glr, lgh_hessian_fn hessian_apply, void *ctx,
                     const lgh_glr_correct_opts_t *opts,
                     lgh_glr_correct_report_t *report);

/* ---- persistence ---------------------------------------------------------
 * Save a built object's spectrum and U (and, with with_extension = 1, the
 * sketch basis and raw projection that lgh_glr_extend continues from) to a
 * file, and restore it against the same B and prior without a rebuild: a
 * restarted serving process, or another process, serves the same model.
 * The reference keeps this state in memory only; the file format is this
 * library's (little-endian, checksummed).  lgh_glr_load checks the size
 * and the checksum (LGH_ERR_ARG_SIZ / LGH_ERR_ARG_WRONG); an object loaded
 * without extension state returns LGH_ERR_ARG_WRONGSTATE from an
 * incremental extend.                                                     */
int lgh_glr_save (const lgh_glr_t *glr, const char *path, int with_extension);
int lgh_glr_load (lgh_Mat B, lgh_prior_t *prior, const char *path,
                  lgh_glr_t **glr);

/* ---- row-sharded operators (more than one GPU) -------------------------
 * The reference distributes vectors and operators over MPI ranks in
 * contiguous row slabs (MPIAIJ; docs/glr-woodbury-formulas.tex:76-98).  A
 * shard plan is one rank's view of a symmetric CSR operator: its owned rows
 * [row0, row1) (the even split r N / P), the remote rows its nonzeros
 * reference (ghosts, ascending, counted per owner rank), and local column
 * indices over an extended row-major block [owned rows; ghost rows].  The
 * caller exchanges the ghost lists (an all-to-all) and registers each
 * peer's requests with lgh_shard_set_sends; per application it packs each
 * peer's rows, sends and receives the contiguous buffers with its own
 * collective (NCCL / gloo) and unpacks them into the ghost rows.  Gram-type
 * products are local products plus an all-reduce; the sketch of rows
 * [i0, i0 + n) is lgh_sketch_rows, identical to those rows of the global
 * sketch (partition-independent, glr_common_impl.h:55-58).             */
typedef struct lgh_shard lgh_shard_t;

void lgh_shard_range (int64_t N, int nranks, int rank, int64_t *row0,
                      int64_t *row1);
/* rowptr (row1 - row0 + 1 entries, rowptr[0] = 0) and colidx (global
 * column indices) of this rank's rows; host arrays, copied.             */
int lgh_shard_create (int64_t N, int nranks, int rank, const int64_t *rowptr,
                      const int32_t *colidx, lgh_shard_t **shard);
int lgh_shard_info (const lgh_shard_t *shard, int64_t *row0, int64_t *row1,
                    int64_t *nghost);
/* borrowed: ghost rows (nghost, ascending) and counts[nranks] per owner   */
int lgh_shard_ghosts (const lgh_shard_t *shard, const int64_t **rows,
                      const int64_t **counts);
/* borrowed: local column indices (one per local nonzero)                 */
int lgh_shard_local_colidx (const lgh_shard_t *shard, const int32_t **colidx);
/* rows (global, owned here) that peer requested as its ghosts            */
int lgh_shard_set_sends (lgh_shard_t *shard, int peer, int64_t count,
                         const int64_t *rows);
/* borrowed: the registered send rows for peer, as local row indices      */
int lgh_shard_sends (const lgh_shard_t *shard, int peer, int64_t *count,
                     const int64_t **local_rows);
/* device: buf (count x w, contiguous) = the send rows of X for peer       */
int lgh_shard_pack (lgh_shard_t *shard, int peer, int w, const double *X,
                    int64_t ldx, double *buf);
/* device: write peer's rows into the ghost rows of Xext (the rows after
 * the nloc owned rows, in ghost order)                                    */
int lgh_shard_unpack (const lgh_shard_t *shard, int peer, int w,
                      const double *buf, double *Xext, int64_t ld);
void lgh_shard_destroy (lgh_shard_t *shard);
/* device: Y[i][j] = randn_at (seed, i0 + i, j0 + j), j < k; zero for
 * k <= j < ld (row-major, leading dimension ld)                          */
int lgh_sketch_rows (uint64_t seed, int64_t i0, int64_t n, int64_t j0, int k,
                     double *Y, int64_t ld);

/* ---- a build over row slabs (one rank per GPU) ---------------------------
 * The reference's MPI layout (docs/glr-woodbury-formulas.tex:76-98): B, Z,
 * the mass lumps and every N-row block are split into contiguous row slabs
 * (rank r owns a contiguous range of rows, ranks in order).  A row-sharded Mat
 * (lgh_mat_create_rows) carries its halo plan and the communicator; a
 * prior made from a row-sharded Z (lgh_prior_create_mat / _pc, with the
 * rank's mass lumps) is a row-sharded prior, and lgh_glr_compute on a
 * row-sharded B and prior builds over the slabs:
 *   - B X and Z X exchange the ghost rows of X once per product (one
 *     all-to-all of the rows each peer references) and multiply the local
 *     rows by [owned rows; ghost rows];
 *   - Z-solves run blocked PCG with two all-reduces of 2 w scalars per
 *     iteration; the preconditioner is rank-local (block Jacobi: the
 *     multigrid V-cycle on the rank's diagonal block of Z, or Jacobi),
 *     so iteration counts grow slowly with the number of ranks and the
 *     solution matches the one-rank solve to the solve tolerance;
 *   - every Gram, Q^T F Q, U^T X and residual norm is the local product
 *     plus one all-reduce (glr_common_impl.h:363, 487, 769, 851); the
 *     small eigenproblem runs replicated, so every rank keeps the same
 *     spectrum and its own rows of U.
 * The sketch is partition-independent (hashed per global row).  Vectors
 * and blocks passed to the object's operations (solve, sample, apply,
 * factor, lgh_glr_get_U) hold the rank's rows; logdet and eigs are
 * replicated.  The batched shift operations, the request loop, the
 * deflation correction and persistence return LGH_ERR_SUP on a
 * row-sharded object.
 *
 * allreduce: buf[0, count) (device, FP64) becomes the elementwise sum over
 * ranks, identical on every rank.  alltoallv: for each peer p, the
 * send_bytes[p] bytes at offset sum_{q<p} send_bytes[q] of send go to p,
 * and the recv_bytes[p] bytes from p land at offset sum_{q<p}
 * recv_bytes[q] of recv (device buffers; recv_bytes[p] equals what p
 * sends here; entries for this rank are 0).  The library synchronises
 * its stream before each call; the callback returns once the data is in
 * place (0), or nonzero to fail the operation with LGH_ERR_GPU.  Every
 * rank makes the same calls in the same order.  The communicator must
 * stay valid for the lifetime of the objects made with it.              */
typedef struct lgh_rows_comm
{
  int    rank, size;
  int  (*allreduce) (double *buf, size_t count, void *ctx);
  int  (*alltoallv) (const void *send, const size_t *send_bytes, void *recv,
                     const size_t *recv_bytes, void *ctx);
  void  *ctx;
}
lgh_rows_comm_t;

/* This rank's rows [row0, row0 + nrows) of a symmetric N x N CSR
 * operator (MatGetOwnershipRange of an MPIAIJ): rowptr (nrows + 1
 * entries, rowptr[0] = 0), global column indices, values; host arrays,
 * copied.  Ranks own contiguous rows in rank order covering [0, N), at
 * least one each (any split: PETSc's layout, or lgh_shard_range's);
 * B and Z of one build must be split alike.  Collective: every rank calls
 * it with its own rows, and all ranks fail together on a bad split.      */
int lgh_mat_create_rows (int64_t N, const lgh_rows_comm_t *comm,
                         int64_t row0, int64_t nrows, const int64_t *rowptr,
                         const int32_t *colidx, const double *vals,
                         lgh_Mat *A);
/* rows of a row-sharded Mat (0 / N / 0 ghosts for an ordinary Mat)       */
int lgh_mat_rows_info (lgh_Mat A, int64_t *row0, int64_t *row1,
                       int64_t *nghost);
/* halo traffic of a row-sharded Mat since its creation: exchanges, bytes
 * this rank sent, seconds in the exchange callback                       */
int lgh_mat_rows_traffic (lgh_Mat A, long *exchanges, int64_t *bytes_sent,
                          double *seconds);
/* `size` communicators for ranks run as threads of one process on one
 * device: the collectives meet on a host barrier (120 s limit, then
 * LGH_ERR_GPU), sum in rank order on the host and copy device to device;
 * no kernel waits for another rank.                                      */
int lgh_rows_local_create (int size, lgh_rows_comm_t *comms);
void lgh_rows_local_destroy (lgh_rows_comm_t *comms);

/* Per-kernel CUDA-event timing of the hot kernels: switch on (1) / off (0)
 * (either resets the figures); read accumulated device milliseconds,
 * launches and algorithmic bytes of kernel id 0 k_pcg_pq, 1 k_pcg_upd,
 * 2 k_cheb (every 8th launch), 3 k_spmm (the B product), 4 k_pcg_init.
 * Returns the kernel's name, NULL past the last id.                     */
int lgh_kernel_timing (int on);
const char *lgh_kernel_timing_get (int id, double *ms, long *launches,
                                   double *bytes);

/* Number of this library's kernel launches since the process started.   */
long lgh_launch_count (void);

/* Host-side runtime counters since the process started: out[0..4] =
 * device allocations, seconds in them, device frees, seconds in them,
 * kernel launches.                                                        */
int lgh_runtime_counters (double *out);

/* Throughput probes (the roofline denominators beside the measured copy
 * bandwidth): out[0..3] = FP64 FMA TFLOP/s, FP32 FMA TFLOP/s, FP64
 * mma.sync TFLOP/s, L2-resident read GB/s.                                */
int lgh_probe_peaks (double *out);

/* Last error message of the calling thread (empty if none).              */
const char *lgh_last_error (void);

/* ---- kernel-level test hooks (host arrays in and out; not used by the
 * build): each runs exactly one device kernel path. ---------------------- */
int lgh_test_sketch (uint64_t seed, int64_t n, int64_t j0, int k,
                     double *out);
int lgh_test_rng_state (uint64_t seed, int64_t n, int64_t j0, int k,
                        uint64_t *out);
int lgh_test_spmm (lgh_Mat A, int w, const double *X, double *Y, int fp32);
/* the same product through the strip form of A at height R (2, 4, 8; 0 =
 * chosen by the cost model); *R_used (nullable) gets the height */
int lgh_test_spmm_strip (lgh_Mat A, int w, const double *X, double *Y,
                         int fp32, int R, int *R_used);
int lgh_test_zsolve (lgh_prior_t *prior, int w, const double *X, double *Y,
                     int fp32);
/* one Chebyshev-Jacobi smoothing step of a square CSR Mat (n x w row-major
 * host blocks) with the smoother's kernel: X in place, Rout = Ro - A d_new,
 * Dout = d_new (flags & 4), d_new = a Do + b D^{-1} Ro (flags & 1: a Do
 * left out; flags & 2: X taken as zero; flags & 8: only Rout written;
 * flags & 16: Do is the residual given to a flags & 8 first step with
 * coefficient bp, whose d and x this step forms).                        */
int lgh_test_cheb_step (lgh_Mat A, int w, double a, double b, int flags,
                        int fp32, double *X, const double *Ro,
                        const double *Do, double *Rout, double *Dout,
                        double bp);
int lgh_test_gram (int64_t n, int w, const double *X, double *G);
int lgh_test_gemm_nn (int64_t n, int k, int m, const double *X,
                      const double *M, double *Y);
int lgh_test_potrf (int n, const double *G, int jitter_mode, double *L,
                    double *Linv, int *info);
int lgh_test_syev (int n, const double *A, double *w, double *V,
                   int *sweeps);
/* The multigrid set-up's first coarsening of a square CSR (host arrays),
 * run on the host alone with no device call: the smoothed-aggregation
 * prolongator P (n x nc) and the symmetrised Galerkin operator
 * Ac = P^T A P (nc x nc), with `threads` OpenMP threads (0: the default).
 * *nc, *p_nnz and *c_nnz always get the sizes; P and Ac are written when
 * p_rowptr / c_rowptr are non-null (n + 1 and nc + 1 row pointers,
 * capacities p_cap / c_cap entries), so a first call with null arrays
 * sizes the second.                                                      */
int lgh_test_mg_galerkin (int64_t n, const int64_t *rowptr,
                          const int32_t *colidx, const double *vals,
                          int threads, int64_t *nc, int64_t *p_rowptr,
                          int32_t *p_colidx, double *p_vals, int64_t p_cap,
                          int64_t *p_nnz, int64_t *c_rowptr,
                          int32_t *c_colidx, double *c_vals, int64_t c_cap,
                          int64_t *c_nnz);

#ifdef __cplusplus
}
#endif

#endif /* LGH_B200_H */
