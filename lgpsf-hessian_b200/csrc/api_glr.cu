/* api_glr.cu -- the GLR object on the device: build, incremental extension
 * and every downstream operation of the reference's replicated backend
 * (include/lgpsf_hessian/impl/glr_common_impl.h:252-1104), with the
 * distributed backend's incremental extension (glr_scalapack_impl.h:
 * 689-915).  All state (B, Z, M, Q, the raw projection A, U, lambda) stays
 * resident in HBM; the host sees only lambda (lgh_glr_eigs) and the report.
 */

#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "lgh_device.cuh"
#include "lgh_internal.h"
#include "lgh_ktime.h"
#include "lgh_objects.h"

namespace lgh
{

/* ---- small device kernels of this file ---------------------------------- */

/* fk[i] = f(lam_i + c) - f(c) for the master formula
 * (glr_common_impl.h:948-966): kind 0: 1/x, 1: x^{-1/2}, 2: x^{1/2},
 * 3: x^p, 4: x (apply after correction), 5: user values f_lam (in fk) */
__global__ void
k_filter_coef (int kept, const double *lam, double c, int kind, double p,
               double fc, double *fk)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kept;
       i += gridDim.x * blockDim.x) {
    const double x = lam[i] + c;
    double f;
    switch (kind) {
    case 0: f = 1. / x; break;
    case 1: f = 1. / pow (x, 0.5); break;
    case 2: f = pow (x, 0.5); break;
    case 3: f = pow (x, p); break;
    case 4: f = x; break;
    default: f = fk[i]; break;
    }
    fk[i] = f - fc;
  }
}

/* W[k + j*kept] *= fk[k] for a kept x m column-major block */
__global__ void
k_scale_rows_cm (int kept, int m, const double *fk, const double *Win,
                 double *Wout)
{
  const int64_t total = (int64_t) kept * m;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x)
    Wout[e] = Win[e] * fk[e % kept];
}

/* batched coefficient block for shift c: D[k + j*kept] = (f(lam_k + c) -
 * f(c)) W[k + j*kept] */
__global__ void
k_shift_coef (int kept, int m, const double *lam, double c, int kind,
              const double *Win, double *Dout)
{
  const int64_t total = (int64_t) kept * m;
  double fc = (kind == 0) ? 1. / c : 1. / sqrt (c);
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int k = (int) (e % kept);
    const double x = lam[k] + c;
    const double f = (kind == 0) ? 1. / x : 1. / sqrt (x);
    Dout[e] = (f - fc) * Win[e];
  }
}

/* sum over kept of log(lam_i + c) - log(c), FP64, one block per shift;
 * compensated (Kahan) per-thread sums, fixed-order tree */
__global__ void
k_logdet (int kept, const double *lam, int nshift, const double *c,
          double *out)
{
  __shared__ double red[256];
  const int sidx = blockIdx.x;
  if (sidx >= nshift) return;
  const double cs = c[sidx], lc = log (cs);
  double s = 0., comp = 0.;
  for (int i = threadIdx.x; i < kept; i += blockDim.x) {
    const double y = (log (lam[i] + cs) - lc) - comp;
    const double t = s + y;
    comp = (t - s) - y;
    s = t;
  }
  red[threadIdx.x] = s;
  __syncthreads ();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads ();
  }
  if (threadIdx.x == 0) out[sidx] = red[0];
}

/* logdet at nshift device-resident shifts into device out[] */
int
launch_logdet (int kept, const double *lam, int nshift, const double *c,
               double *out, cudaStream_t s)
{
  k_logdet<<<nshift, 256, 0, s>>> (kept, lam, nshift, c, out);
  LGH_LAUNCH_CHECK ();
  return 0;
}

/* T = (A + A^T)/2 (glr_common_impl.h:490-494) */
__global__ void
k_symmetrize (int n, const double *A, double *T)
{
  const int64_t nn = (int64_t) n * n;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < nn;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int i = (int) (e % n), j = (int) (e / n);
    T[e] = (i == j) ? A[e] : 0.5 * (A[e] + A[j + (size_t) i * n]);
  }
}

/* grow the raw projection by symmetry (glr_scalapack_impl.h:819-840):
 * A2 (l2 x l2) from A (l1 x l1) and Cnew = Q_all^T F Q_new (l2 x k) */
__global__ void
k_grow_A (int l1, int l2, const double *A, const double *Cn, double *A2)
{
  const int64_t nn = (int64_t) l2 * l2;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < nn;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int i = (int) (e % l2), j = (int) (e / l2);
    double v;
    if (j < l1 && i < l1) v = A[i + (size_t) j * l1];
    else if (j < l1) v = Cn[j + (size_t) (i - l1) * l2];
    else v = Cn[i + (size_t) (j - l1) * l2];
    A2[e] = v;
  }
}

/* lraw[j] = w[order[j]], j < kept */
__global__ void
k_gather_raw (int kept, const double *w, const int *order, double *lraw)
{
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < kept;
       j += gridDim.x * blockDim.x)
    lraw[j] = w[order[j]];
}

static int
sgrid (int64_t total)
{
  int64_t g = (total + 255) / 256;
  if (g < 1) g = 1;
  if (g > num_sms () * 8) g = num_sms () * 8;
  return (int) g;
}

/* ---- ell x ell scratch of one build / extension ------------------------- */

struct Small
{
  int n = 0;
  DBuf<double> G, G0, M, T, A2, V, V2, w, C, work, sel, lam;
  DBuf<int> order, info;
  int alloc (int n_, int64_t rows, int maxw)
  {
    n = n_;
    const size_t nn = (size_t) n * n;
    LGH_TRY (G.alloc (nn));
    LGH_TRY (G0.alloc (nn));
    LGH_TRY (M.alloc (nn));
    LGH_TRY (T.alloc (nn));
    LGH_TRY (A2.alloc (nn));
    LGH_TRY (V.alloc (nn));
    LGH_TRY (V2.alloc (nn));
    LGH_TRY (w.alloc (n));
    LGH_TRY (C.alloc (nn));
    /* split-K workspace: enough for every (m1, m2) <= (maxw, maxw) shape */
    LGH_TRY (work.alloc (std::max (gemm_tn_work_elems (rows, maxw, maxw),
                                   gemm_tn_work_max (maxw, maxw))));
    LGH_TRY (sel.alloc (8));
    LGH_TRY (lam.alloc (n));
    LGH_TRY (order.alloc (n));
    LGH_TRY (info.alloc (4));
    return 0;
  }
};

/* ---- the operator F ------------------------------------------------------ */

/* Y = F X = M^{1/2} Z^{-1} B Z^{-T} M^{1/2} X (glr_common_impl.h:316-336);
 * W is scratch of the same shape; the row scalings are fused into the
 * Z-solves' load and store. */
template <typename T>
static int
apply_F (lgh_glr_t *g, int w, const T *X, int ldx, T *Y, int ldy, T *W,
         int ldw)
{
  cudaStream_t s = stream ();
  const double *ms = g->prior->msqrt.p;
  /* FP32 blocks: the prior's tolerance unless inner_rtol asks for a looser
   * one (inner_rtol <= 0: the prior's) */
  const double rt = std::is_same<T, float>::value && g->exec.inner_rtol > 0.
                    ? std::max (g->exec.inner_rtol, g->prior->zcfg.rtol) : 0.;
  double t0 = wall ();
  LGH_TRY (prior_solve_rows<T> (g->prior, w, X, ldx, ms, W, ldw, nullptr, rt));
  double t1 = wall ();
  static thread_local EventRing ring;
  const bool timing = ktime_on ();
  LGH_TRY (mat_prepare_block (g->B, w));   /* once per operator */
  if (timing) LGH_TRY (ring.record (s));
  LGH_TRY (mat_mult_block<T> (g->B, W, ldw, Y, ldy, w, s));
  if (timing) LGH_TRY (ring.record (s));
  LGH_CUDA (cudaStreamSynchronize (s));
  if (timing) {
    const double bytes = (double) g->B->csr.nnz * (sizeof (T) + 4)
                         + 8. * (g->n + 1) + 2. * g->n * w * sizeof (T);
    LGH_TRY (ring.drain ({ K_SPMM }, { bytes }));
  }
  double t2 = wall ();
  LGH_TRY (prior_solve_rows<T> (g->prior, w, Y, ldy, nullptr, Y, ldy, ms, rt));
  LGH_CUDA (cudaStreamSynchronize (s));
  double t3 = wall ();
  g->stats.t_zsolve += (t1 - t0) + (t3 - t2);
  g->stats.t_spmm += t2 - t1;
  return 0;
}

/* X <- X L^{-T}, twice (CholQR2, glr_common_impl.h:370-407); the result
 * returns to X, Tmp is scratch.  jitter_mode 0 = replicated rule.  rc
 * (row slabs): the Gram of the local rows is all-reduced before the
 * factorisation, which every rank then repeats identically. */
template <typename T>
static int
cholqr2 (int64_t n, int w, T *X, int ldx, T *Tmp, int ldt, Small &sm,
         int jitter_mode, int *jittered, const lgh_rows_comm_t *rc = nullptr)
{
  cudaStream_t s = stream ();
  for (int pass = 0; pass < 2; pass++) {
    T *src = pass == 0 ? X : Tmp;
    T *dst = pass == 0 ? Tmp : X;
    const int lds = pass == 0 ? ldx : ldt, ldd = pass == 0 ? ldt : ldx;
    LGH_TRY (launch_gemm_tn<T> (n, w, w, src, lds, src, lds, sm.G.p, w, 0,
                                sm.work.p, sm.work.n, s));
    if (rc) LGH_TRY (rows_allreduce (*rc, sm.G.p, (size_t) w * w, s));
    LGH_TRY (launch_potrf (w, sm.G.p, sm.G0.p, jitter_mode, sm.info.p, s));
    int info[2];
    LGH_CUDA (cudaMemcpyAsync (info, sm.info.p, 2 * sizeof (int),
                               cudaMemcpyDeviceToHost, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    LGH_CHECK (info[0] == 0, LGH_ERR_LIB, "cholqr2: potrf failed twice");
    if (jittered) *jittered += info[1];
    LGH_TRY (launch_trtri_lower (w, sm.G.p, sm.M.p, 1, s));
    LGH_TRY (launch_gemm_nn<T> (n, w, w, 1.0, src, lds, sm.M.p, w, 0.,
                                (const T *) nullptr, 0, dst, ldd, s));
  }
  return 0;
}

/* panel CholQR2 with the distributed backend's jitter
 * (glr_scalapack_impl.h:110-148), in place via Tmp (>= n x bw) */
template <typename T>
static int
panel_cholqr (int64_t n, int bw, T *P, int ldp, T *Tmp, int ldt, Small &sm,
              const lgh_rows_comm_t *rc)
{
  LGH_TRY (cholqr2<T> (n, bw, P, ldp, Tmp, ldt, sm, 1, nullptr, rc));
  return 0;
}

/* BCGS2: orthonormalise columns [p_start, ell) of Y against [0, p_start)
 * and each other, in panels of b (glr_scalapack_impl.h:153-195) */
template <typename T>
static int
bcgs2 (int64_t n, T *Y, int ld, int ell, int b, int p_start, T *Tmp,
       int ldt, Small &sm, const lgh_rows_comm_t *rc)
{
  cudaStream_t s = stream ();
  for (int p0 = p_start; p0 < ell; p0 += b) {
    const int bw = std::min (b, ell - p0);
    T *pa = Y + p0;
    for (int sweep = 0; sweep < 2; sweep++) {
      if (p0 > 0) {
        /* C = Y(:, 0:p0)^T P ; P -= Y(:, 0:p0) C */
        LGH_TRY (launch_gemm_tn<T> (n, p0, bw, Y, ld, pa, ld, sm.C.p, p0, 0,
                                    sm.work.p, sm.work.n, s));
        if (rc) LGH_TRY (rows_allreduce (*rc, sm.C.p, (size_t) p0 * bw, s));
        LGH_TRY (launch_gemm_nn<T> (n, p0, bw, -1.0, Y, ld, sm.C.p, p0, 1.0,
                                    pa, ld, pa, ld, s));
      }
      LGH_TRY (panel_cholqr<T> (n, bw, pa, ld, Tmp, ldt, sm, rc));
    }
  }
  return 0;
}

/* eigensolve of sym(A) + selection + U = Q C_kept + report
 * (glr_common_impl.h:469-574) */
template <typename T>
static int
rayleigh_ritz (lgh_glr_t *g, int ell, const T *Q, int ldq, const double *Araw,
               Small &sm, lgh_glr_report_t *rep)
{
  cudaStream_t s = stream ();
  const int64_t n = g->n;
  double t0 = wall ();
  k_symmetrize<<<sgrid ((int64_t) ell * ell), 256, 0, s>>> (ell, Araw, sm.T.p);
  LGH_LAUNCH_CHECK ();
  int sweeps = 0;
  LGH_TRY (launch_syev_jacobi (ell, sm.T.p, sm.V.p, sm.w.p, sm.A2.p, sm.V2.p,
                               &sweeps, s));
  LGH_TRY (launch_select (ell, sm.w.p, sm.V.p, g->opts.trunc_abs,
                          g->opts.trunc_rel, (int) g->opts.treat, sm.order.p,
                          sm.sel.p, sm.lam.p, sm.C.p, s));
  double sel[6];
  LGH_CUDA (cudaMemcpyAsync (sel, sm.sel.p, 6 * sizeof (double),
                             cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  int kept = (int) sel[0];
  if (g->exec.rank_cap > 0 && kept > g->exec.rank_cap) {
    /* rank r with oversampling: keep the r largest |lambda|; the first
     * mode cut by the cap becomes next_abs */
    kept = g->exec.rank_cap;
    double nxt = 0.;
    LGH_CUDA (cudaMemcpy (&nxt, sm.lam.p + kept, sizeof (double),
                          cudaMemcpyDeviceToHost));
    sel[2] = fabs (nxt);
  }
  rep->kept = kept;
  rep->lam_abs_max = sel[1];
  rep->next_abs = sel[2];
  rep->lam_raw_min = sel[3];
  rep->lam_raw_max = sel[4];
  rep->n_negative_raw = (int) sel[5];
  double t1 = wall ();
  rep->t_dense += t1 - t0;
  g->stats.t_eig += t1 - t0;

  g->kept = kept;
  g->ldu = round_ld (std::max (kept, 1));
  g->lam_h.assign (std::max (kept, 1), 0.);
  LGH_TRY (g->lam_d.alloc (std::max (kept, 1)));
  LGH_TRY (g->lraw_d.alloc (std::max (kept, 1)));
  if (kept > 0) {
    LGH_CUDA (cudaMemcpyAsync (g->lam_h.data (), sm.lam.p, kept * sizeof (double),
                               cudaMemcpyDeviceToHost, s));
    LGH_CUDA (cudaMemcpyAsync (g->lam_d.p, sm.lam.p, kept * sizeof (double),
                               cudaMemcpyDeviceToDevice, s));
    k_gather_raw<<<1, 256, 0, s>>> (kept, sm.w.p, sm.order.p, g->lraw_d.p);
    LGH_LAUNCH_CHECK ();
  }
  g->have_wz = 0;
  LGH_TRY (g->U.alloc ((size_t) n * g->ldu));
  LGH_CUDA (cudaMemsetAsync (g->U.p, 0, (size_t) n * g->ldu * sizeof (double), s));
  if (kept > 0) {
    if constexpr (std::is_same<T, double>::value) {
      LGH_TRY (launch_gemm_nn<double> (n, ell, kept, 1.0, Q, ldq, sm.C.p, ell,
                                       0., (const double *) nullptr, 0, g->U.p,
                                       g->ldu, s));
    } else {
      LGH_TRY (g->U32.alloc ((size_t) n * g->ldu));
      LGH_TRY (launch_gemm_nn<float> (n, ell, kept, 1.0, Q, ldq, sm.C.p, ell,
                                      0., (const float *) nullptr, 0, g->U32.p,
                                      g->ldu, s));
      LGH_TRY (launch_f32_to_f64 (n, kept, g->U32.p, g->ldu, g->U.p, g->ldu, s));
    }
  }
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

/* Y = F X over w columns on a column-sharded object: this rank applies F
 * to its own columns, then one all-gather of the packed column blocks
 * rebuilds all w columns of Y on every rank (one device: plain apply_F) */
template <typename T>
static int
apply_F_cols (lgh_glr_t *g, int w, const T *X, int ldx, T *Y, int ldy, T *W,
              int ldw)
{
  const lgh_comm_t &cm = g->comm;
  if (cm.size <= 1) return apply_F<T> (g, w, X, ldx, Y, ldy, W, ldw);
  cudaStream_t s = stream ();
  const int64_t n = g->n;
  int c0, c1, wmax = 0;
  for (int r = 0; r < cm.size; r++) {
    lgh_cols_range (w, r, cm.size, &c0, &c1);
    wmax = std::max (wmax, c1 - c0);
  }
  lgh_cols_range (w, cm.rank, cm.size, &c0, &c1);
  if (c1 > c0)
    LGH_TRY (apply_F<T> (g, c1 - c0, X + c0, ldx, Y + c0, ldy, W + c0, ldw));
  const int ldp = round_ld (std::max (wmax, 1));
  const size_t len = (size_t) n * ldp * sizeof (T);
  char *snd = (char *) cm.send, *rcv = (char *) cm.recv;
  if (!snd || !rcv || cm.bytes < len) {
    LGH_TRY (g->xsend.alloc (len));
    LGH_TRY (g->xrecv.alloc (len * cm.size));
    snd = g->xsend.p;
    rcv = g->xrecv.p;
  }
  if (c1 > c0)
    LGH_TRY (launch_copy_block<T> (n, c1 - c0, Y + c0, ldy, (T *) snd, ldp, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  LGH_CHECK (cm.allgather (snd, rcv, len, cm.ctx) == 0, LGH_ERR_GPU,
             "column-sharded build: the all-gather failed (rank %d of %d)",
             cm.rank, cm.size);
  for (int r = 0; r < cm.size; r++) {
    if (r == cm.rank) continue;
    int r0, r1;
    lgh_cols_range (w, r, cm.size, &r0, &r1);
    if (r1 > r0)
      LGH_TRY (launch_copy_block<T> (n, r1 - r0, (const T *) (rcv + r * len),
                                     ldp, Y + r0, ldy, s));
  }
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

/* max_j || F u_j - lam_raw_j u_j || (glr_common_impl.h:576-600).  FY, C
 * (nullable): the projection pass's block F Q (n x ell, ld ldf) and the
 * kept Ritz coefficients (ell x kept, column-major): F U = (F Q) C, one
 * product, instead of another F-apply of U (check_form) */
template <typename T>
static int
residual_check (lgh_glr_t *g, T *Ubuf, T *FU, T *Wk, lgh_glr_report_t *rep,
                const T *FY = nullptr, int ldf = 0, const double *C = nullptr,
                int ell = 0)
{
  if (!g->opts.check || g->kept == 0) return 0;
  cudaStream_t s = stream ();
  const int kept = g->kept, ldu = g->ldu;
  double t0 = wall ();
  if (FY && C && g->exec.check_form == LGH_CHECK_PROJ) {
    LGH_TRY (launch_gemm_nn<T> (g->n, ell, kept, 1.0, FY, ldf, C, ell, 0.,
                                FU, ldu, FU, ldu, s));
  } else {
    LGH_TRY (apply_F_cols<T> (g, kept, Ubuf, ldu, FU, ldu, Wk, ldu));
    rep->t_operator += wall () - t0;
  }
  DBuf<double> norms, part;
  DBuf<unsigned> cnt;
  LGH_TRY (norms.alloc (kept));
  LGH_TRY (part.alloc ((size_t) kept * num_sms () * 2));
  LGH_TRY (cnt.alloc (2));
  LGH_CUDA (cudaMemsetAsync (cnt.p, 0, 2 * sizeof (unsigned), s));
  LGH_TRY (launch_resid_norms<T> (g->n, kept, FU, ldu, Ubuf, ldu, g->lraw_d.p,
                                  norms.p, part.p, cnt.p, s));
  std::vector<double> h (kept);
  LGH_CUDA (cudaMemcpyAsync (h.data (), norms.p, kept * sizeof (double),
                             cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  if (g->rows) {
    /* row slabs: the squared local norms summed over ranks */
    for (double &v : h) v *= v;
    LGH_CUDA (cudaMemcpy (norms.p, h.data (), kept * sizeof (double),
                          cudaMemcpyHostToDevice));
    LGH_TRY (rows_allreduce (*g->rows, norms.p, kept, s));
    LGH_CUDA (cudaMemcpy (h.data (), norms.p, kept * sizeof (double),
                          cudaMemcpyDeviceToHost));
    for (double &v : h) v = sqrt (v);
  }
  double mx = 0.;
  for (double v : h) mx = std::max (mx, v);
  rep->resid_max = mx;
  g->stats.t_check += wall () - t0;
  return 0;
}

/* the replicated build (glr_common_impl.h:414-608) on the device */
template <typename T>
static int
build (lgh_glr_t *g, lgh_glr_report_t *rep)
{
  cudaStream_t s = stream ();
  const int ell = g->opts.ell;
  const int ld = round_ld (ell);
  const int64_t n = g->n;
  memset (rep, 0, sizeof (*rep));
  const double tb = wall ();
  DBuf<T> Q, Y, W;
  LGH_TRY (Q.alloc ((size_t) n * ld));
  LGH_TRY (Y.alloc ((size_t) n * ld));
  LGH_TRY (W.alloc ((size_t) n * ld));
  Small sm;
  LGH_TRY (sm.alloc (ell, n, ell));

  /* Omega, hashed per (seed, global row, column) */
  double t0 = wall ();
  if constexpr (std::is_same<T, double>::value)
    LGH_TRY (launch_sketch (g->opts.seed, n, 0, ell, Q.p, ld, s, g->row0));
  else
    LGH_TRY (launch_sketch_f32 (g->opts.seed, n, 0, ell, Q.p, ld, s, g->row0));
  LGH_CUDA (cudaStreamSynchronize (s));
  g->stats.t_sketch += wall () - t0;

  /* Y = F Omega; power passes with re-orthonormalisation */
  t0 = wall ();
  LGH_TRY (apply_F_cols<T> (g, ell, Q.p, ld, Y.p, ld, W.p, ld));
  rep->t_operator += wall () - t0;
  for (int p = 0; p < g->opts.q_power; p++) {
    t0 = wall ();
    LGH_TRY (cholqr2<T> (n, ell, Y.p, ld, W.p, ld, sm, 0, nullptr, g->rows));
    LGH_CUDA (cudaStreamSynchronize (s));
    double dt = wall () - t0;
    rep->t_dense += dt;
    g->stats.t_orth += dt;
    Q.swap (Y);
    t0 = wall ();
    LGH_TRY (apply_F_cols<T> (g, ell, Q.p, ld, Y.p, ld, W.p, ld));
    rep->t_operator += wall () - t0;
  }
  t0 = wall ();
  LGH_TRY (cholqr2<T> (n, ell, Y.p, ld, W.p, ld, sm, 0, nullptr, g->rows));
  LGH_CUDA (cudaStreamSynchronize (s));
  {
    double dt = wall () - t0;
    rep->t_dense += dt;
    g->stats.t_orth += dt;
  }
  Q.swap (Y); /* Q orthonormal */

  /* T = Q^T F Q */
  t0 = wall ();
  LGH_TRY (apply_F_cols<T> (g, ell, Q.p, ld, Y.p, ld, W.p, ld));
  rep->t_operator += wall () - t0;
  DBuf<double> A;
  LGH_TRY (A.alloc ((size_t) ell * ell));
  LGH_TRY (launch_gemm_tn<T> (n, ell, ell, Q.p, ld, Y.p, ld, A.p, ell, 0,
                              sm.work.p, sm.work.n, s));
  if (g->rows) LGH_TRY (rows_allreduce (*g->rows, A.p, (size_t) ell * ell, s));
  LGH_TRY (rayleigh_ritz<T> (g, ell, Q.p, ld, A.p, sm, rep));

  /* residual check on the kept columns (U in FP64 or FP32 blocks) */
  if (g->opts.check && g->kept > 0) {
    /* Y still holds F Q and sm.C the kept coefficients: the projection
     * form writes F U = Y C into W; the apply form overwrites Y with F U
     * and uses W as its scratch */
    T *FU = g->exec.check_form == LGH_CHECK_PROJ ? W.p : Y.p;
    if constexpr (std::is_same<T, double>::value)
      LGH_TRY (residual_check<double> (g, g->U.p, FU, W.p, rep, Y.p, ld,
                                       sm.C.p, ell));
    else
      LGH_TRY (residual_check<float> (g, g->U32.p, FU, W.p, rep, Y.p, ld,
                                      sm.C.p, ell));
  }

  /* keep the sketch state for the incremental extension */
  g->ell = ell;
  g->ldq = ld;
  if (g->opts.backend != LGH_GLR_REPLICATED) {
    if constexpr (std::is_same<T, double>::value) g->Q.swap (Q);
    else g->Q32.swap (Q);
    g->A.swap (A);
  }
  g->stats.t_build += wall () - tb;
  return 0;
}

/* incremental extension (glr_scalapack_impl.h:689-915), U materialised */
template <typename T>
static int
extend_incremental (lgh_glr_t *g, int k_new, lgh_glr_report_t *rep)
{
  cudaStream_t s = stream ();
  const int64_t n = g->n;
  const int l1 = g->ell, l2 = l1 + k_new;
  const int ld1 = g->ldq, ld2 = round_ld (l2), ldk = round_ld (k_new);
  const int panel = g->opts.panel > 0 ? g->opts.panel : 64;
  memset (rep, 0, sizeof (*rep));
  const double tb = wall ();
  T *Qold;
  if constexpr (std::is_same<T, double>::value) Qold = g->Q.p;
  else Qold = g->Q32.p;
  LGH_CHECK (Qold != nullptr && g->A.p != nullptr, LGH_ERR_ARG_WRONGSTATE,
             "lgh_glr_extend: no sketch state kept");
  DBuf<T> Qb, Qn, Yn, Wn;
  LGH_TRY (Qb.alloc ((size_t) n * ld2));
  LGH_TRY (Qn.alloc ((size_t) n * ldk));
  LGH_TRY (Yn.alloc ((size_t) n * ldk));
  LGH_TRY (Wn.alloc ((size_t) n * std::max (ldk, ld2)));
  Small sm;
  LGH_TRY (sm.alloc (l2, n, l2));
  LGH_CUDA (cudaMemsetAsync (Qb.p, 0, (size_t) n * ld2 * sizeof (T), s));
  LGH_TRY (launch_copy_block<T> (n, l1, Qold, ld1, Qb.p, ld2, s));
  double t0 = wall ();
  if constexpr (std::is_same<T, double>::value)
    LGH_TRY (launch_sketch (g->opts.seed, n, l1, k_new, Qn.p, ldk, s, g->row0));
  else
    LGH_TRY (launch_sketch_f32 (g->opts.seed, n, l1, k_new, Qn.p, ldk, s, g->row0));
  LGH_CUDA (cudaStreamSynchronize (s));
  g->stats.t_sketch += wall () - t0;

  /* power passes on the new block (internal orthonormalisation only) */
  t0 = wall ();
  LGH_TRY (apply_F_cols<T> (g, k_new, Qn.p, ldk, Yn.p, ldk, Wn.p, ldk));
  rep->t_operator += wall () - t0;
  for (int p = 0; p < g->opts.q_power; p++) {
    t0 = wall ();
    LGH_TRY (bcgs2<T> (n, Yn.p, ldk, k_new, panel, 0, Wn.p, ldk, sm, g->rows));
    LGH_CUDA (cudaStreamSynchronize (s));
    rep->t_dense += wall () - t0;
    Qn.swap (Yn);
    t0 = wall ();
    LGH_TRY (apply_F_cols<T> (g, k_new, Qn.p, ldk, Yn.p, ldk, Wn.p, ldk));
    rep->t_operator += wall () - t0;
  }
  /* F^{q+1} Omega_new into Qb's new columns; BCGS2 vs old + internal */
  LGH_TRY (launch_copy_block<T> (n, k_new, Yn.p, ldk, Qb.p + l1, ld2, s));
  t0 = wall ();
  LGH_TRY (bcgs2<T> (n, Qb.p, ld2, l2, panel, l1, Wn.p, ld2, sm, g->rows));
  LGH_CUDA (cudaStreamSynchronize (s));
  rep->t_dense += wall () - t0;
  /* F Q_new, border columns Cnew = Q_all^T (F Q_new) */
  LGH_TRY (launch_copy_block<T> (n, k_new, Qb.p + l1, ld2, Qn.p, ldk, s));
  t0 = wall ();
  LGH_TRY (apply_F_cols<T> (g, k_new, Qn.p, ldk, Yn.p, ldk, Wn.p, ldk));
  rep->t_operator += wall () - t0;
  DBuf<double> Cn, A2;
  LGH_TRY (Cn.alloc ((size_t) l2 * k_new));
  LGH_TRY (A2.alloc ((size_t) l2 * l2));
  LGH_TRY (launch_gemm_tn<T> (n, l2, k_new, Qb.p, ld2, Yn.p, ldk, Cn.p, l2, 0,
                              sm.work.p, sm.work.n, s));
  if (g->rows) LGH_TRY (rows_allreduce (*g->rows, Cn.p, (size_t) l2 * k_new, s));
  k_grow_A<<<sgrid ((int64_t) l2 * l2), 256, 0, s>>> (l1, l2, g->A.p, Cn.p, A2.p);
  LGH_LAUNCH_CHECK ();
  g->opts.ell = l2;
  LGH_TRY (rayleigh_ritz<T> (g, l2, Qb.p, ld2, A2.p, sm, rep));
  g->ell = l2;
  g->ldq = ld2;
  if constexpr (std::is_same<T, double>::value) g->Q.swap (Qb);
  else g->Q32.swap (Qb);
  g->A.swap (A2);
  g->stats.t_build += wall () - tb;
  return 0;
}

/* ---- downstream ---------------------------------------------------------- */

static int
glr_scratch (lgh_glr_t *g)
{
  LGH_TRY (g->w1.alloc (g->n));
  LGH_TRY (g->w2.alloc (g->n));
  LGH_TRY (g->wk.alloc (std::max (g->kept, 1) + 8));
  LGH_TRY (g->fk.alloc (std::max (g->kept, 1) + 8));
  LGH_TRY (g->part.alloc (std::max<size_t> (gemm_tn_work_elems (g->n, std::max (g->kept, 1), 1), 64)));
  return 0;
}

/* out = f_c in + U diag(f_lam - f_c) U^T in  (glr_common_impl.h:948-966);
 * coefficients from kind (see k_filter_coef) or user values f_user */
static int
filter_core (lgh_glr_t *g, int kind, double c, double p, const double *f_user,
             double f_c, const double *in, double *out)
{
  cudaStream_t s = stream ();
  const int64_t n = g->n;
  if (g->kept == 0) return launch_vec_scale (n, in, nullptr, f_c, out, s);
  LGH_TRY (glr_scratch (g));
  if (kind == 5)
    LGH_CUDA (cudaMemcpyAsync (g->fk.p, f_user, g->kept * sizeof (double),
                               cudaMemcpyHostToDevice, s));
  k_filter_coef<<<1, 256, 0, s>>> (g->kept, g->lam_d.p, c, kind, p, f_c, g->fk.p);
  LGH_LAUNCH_CHECK ();
  LGH_TRY (launch_gemm_tn<double> (n, g->kept, 1, g->U.p, g->ldu, in, 1,
                                   g->wk.p, g->kept, 0, g->part.p, g->part.n, s));
  if (g->rows) LGH_TRY (rows_allreduce (*g->rows, g->wk.p, g->kept, s));
  k_scale_rows_cm<<<1, 256, 0, s>>> (g->kept, 1, g->fk.p, g->wk.p, g->wk.p);
  LGH_LAUNCH_CHECK ();
  LGH_TRY (launch_gemm_nn<double> (n, g->kept, 1, 1.0, g->U.p, g->ldu, g->wk.p,
                                   g->kept, f_c, in, 1, out, 1, s));
  return 0;
}

static int
check_shift (lgh_glr_t *g, double c, const char *who)
{
  LGH_CHECK (c > g->floor, LGH_ERR_ARG_OUTOFRANGE,
             "%s: shift c must exceed the spectrum floor %g", who, g->floor);
  return 0;
}

static int
check_vecs (lgh_glr_t *g, lgh_Vec a, lgh_Vec b, const char *who)
{
  LGH_CHECK (g && a && b, LGH_ERR_ARG_NULL, "%s: NULL argument", who);
  LGH_CHECK (a->n == g->n && b->n == g->n, LGH_ERR_ARG_SIZ, "%s: size", who);
  LGH_CHECK (a->d != b->d, LGH_ERR_ARG_WRONG, "%s: in/out alias", who);
  return 0;
}

/* the FP64 Z-solves of the downstream block operations: FP64 PCG with an
 * FP64 V-cycle, or for a mixed-precision object with an FP32 V-cycle;
 * both to the prior's tolerance.  X and Y must not overlap. */
static int
glr_zsolve (lgh_glr_t *g, int w, const double *X, int ldx, const double *s_in,
            double *Y, int ldy, const double *s_out)
{
  if (g->exec.precision == LGH_PREC_MIXED)
    return prior_solve_pc32 (g->prior, w, X, ldx, s_in, Y, ldy, s_out);
  return prior_solve_rows<double> (g->prior, w, X, ldx, s_in, Y, ldy, s_out);
}

/* W = Z^{-1} M^{1/2} U, once per build (the shift-independent precompute of
 * the batched operations) */
int
ensure_wz (lgh_glr_t *g)
{
  if (g->have_wz || g->kept == 0) return 0;
  LGH_TRY (g->Wz.alloc ((size_t) g->n * g->ldu));
  LGH_CUDA (cudaMemsetAsync (g->Wz.p, 0, (size_t) g->n * g->ldu * sizeof (double), stream ()));
  LGH_TRY (glr_zsolve (g, g->kept, g->U.p, g->ldu, g->prior->msqrt.p, g->Wz.p,
                       g->ldu, nullptr));
  g->have_wz = 1;
  return 0;
}

/* batched solve (kind 0) or sample (kind 1) */
static int
batch_op (lgh_glr_t *g, int kind, int nshift, const double *c, int m,
          const double *rhs, int64_t ldr, double *x, int64_t ldx)
{
  cudaStream_t s = stream ();
  const int64_t n = g->n;
  LGH_CHECK (g && c && rhs && x, LGH_ERR_ARG_NULL, "batch: NULL argument");
  LGH_CHECK (!g->rows, LGH_ERR_SUP,
             "batch: a row-sharded object runs the per-shift operations");
  LGH_CHECK (m > 0 && nshift > 0 && ldr >= n && ldx >= n, LGH_ERR_ARG_SIZ, "batch: size");
  std::vector<double> ch (nshift);
  LGH_CUDA (cudaMemcpy (ch.data (), c, nshift * sizeof (double), cudaMemcpyDefault));
  for (int i = 0; i < nshift; i++) LGH_TRY (check_shift (g, ch[i], "batch"));
  /* one shift and no W yet: the per-call formula of glr_common_impl.h:
   * 1007-1024 / 1084-1091 (the same Z-solves of width m, no W) */
  const bool direct = nshift == 1 && !g->have_wz && g->kept > 0;
  if (!direct) LGH_TRY (ensure_wz (g));
  const int ldm = round_ld (m), kept = g->kept;
  const double *ms = g->prior->msqrt.p;
  if (direct) {
    DBuf<double> R, Y0, Xs, Wc, Dc, work;
    LGH_TRY (R.alloc ((size_t) n * ldm));
    LGH_TRY (Y0.alloc ((size_t) n * ldm));
    LGH_TRY (Xs.alloc ((size_t) n * ldm));
    LGH_TRY (Wc.alloc ((size_t) std::max (kept, 1) * m));
    LGH_TRY (Dc.alloc ((size_t) std::max (kept, 1) * m));
    LGH_TRY (work.alloc (std::max<size_t> (gemm_tn_work_elems (n, std::max (kept, 1), m), 64)));
    LGH_TRY (launch_colmajor_to_rowmajor (n, m, rhs, ldr, R.p, ldm, nullptr, s));
    if (kind == 0) {
      /* r2 = M^{1/2} Z^{-1} r (into R) */
      LGH_TRY (glr_zsolve (g, m, R.p, ldm, nullptr, Xs.p, ldm, ms));
      R.swap (Xs);
    }
    LGH_TRY (launch_gemm_tn<double> (n, kept, m, g->U.p, g->ldu, R.p, ldm, Wc.p,
                                     kept, 0, work.p, work.n, s));
    /* t = f(c) r2 + U diag(f(lam + c) - f(c)) U^T r2, x = Z^{-1} M^{1/2} t */
    const double cs = ch[0];
    const double fc = (kind == 0) ? 1. / cs : 1. / sqrt (cs);
    k_shift_coef<<<sgrid ((int64_t) kept * m), 256, 0, s>>> (kept, m, g->lam_d.p, cs,
                                                            kind, Wc.p, Dc.p);
    LGH_LAUNCH_CHECK ();
    LGH_TRY (launch_gemm_nn<double> (n, kept, m, 1.0, g->U.p, g->ldu, Dc.p, kept, fc,
                                     R.p, ldm, Xs.p, ldm, s));
    LGH_TRY (glr_zsolve (g, m, Xs.p, ldm, ms, Y0.p, ldm, nullptr));
    LGH_TRY (launch_rowmajor_to_colmajor (n, m, Y0.p, ldm, x, ldx, nullptr, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    return 0;
  }
  /* the shift-independent part: r2 (solve: M^{1/2} Z^{-1} r; sample: xi),
   * C = U^T r2 and y0 = Z^{-1} M^{1/2} r2, in the object's batch plan */
  ShiftPlan *P = nullptr;
  LGH_TRY (shift_plan_get (g, n, m, kept, nshift, &P));
  double *R = shift_plan_R (P), *Xs = shift_plan_Xs (P);
  double *Y0 = shift_plan_Y0 (P), *Wc = shift_plan_Wc (P);
  size_t wn = 0;
  double *work = shift_plan_work (P, &wn);
  LGH_TRY (launch_colmajor_to_rowmajor (n, m, rhs, ldr, R, ldm, nullptr, s));
  double *r2 = R;
  if (kind == 0) {
    LGH_TRY (glr_zsolve (g, m, R, ldm, nullptr, Xs, ldm, ms));
    r2 = Xs;
  }
  if (kept > 0)
    LGH_TRY (launch_gemm_tn<double> (n, kept, m, g->U.p, g->ldu, r2, ldm, Wc,
                                     kept, 0, work, wn, s));
  LGH_TRY (glr_zsolve (g, m, r2, ldm, ms, Y0, ldm, nullptr));
  /* every shift in one fused launch (a captured graph after the first
   * call of a shape); the tile variant is the autotuner's */
  struct Trial
  {
    ShiftPlan *P;
    lgh_glr_t *g;
    int kind, nshift, m;
    const double *c;
    double *x;
    int64_t ldx;
    static int run (int v, void *ctx)
    {
      Trial *t = (Trial *) ctx;
      return shift_plan_run_eager (t->P, t->g, t->kind, t->nshift, t->c, t->m,
                                   t->x, t->ldx, v);
    }
  } trial{ P, g, kind, nshift, m, ch.data (), x, ldx };
  /* mixed-precision objects: the tcgen05 (TF32 x 3) form; FP64 objects:
   * the FP64 tensor-core form */
  const bool tc = g->exec.precision == LGH_PREC_MIXED && kept > 0
                  && umma_supported ();
  if (tc) LGH_TRY (shift_plan_prepare_umma (P, g, nshift, m));
  struct Offset
  {
    Trial *t;
    int base;
    static int run (int v, void *ctx)
    {
      Offset *o = (Offset *) ctx;
      return Trial::run (o->base + v, o->t);
    }
  } off{ &trial, tc ? kShiftVariants : 0 };
  int v = 0, measured = 0;
  LGH_TRY (tune_pick (tc ? "shift_combine_tf32x3" : "shift_combine_f64", n,
                      kept, m, nshift, tc ? kUmmaVariants : kShiftVariants,
                      &Offset::run, &off, &v, &measured));
  const int variant = off.base + v;
  /* a measured first call has its result from the trials already */
  if (!measured)
    LGH_TRY (shift_plan_combine (P, g, kind, nshift, ch.data (), m, x, ldx,
                                 variant));
  LGH_CUDA (cudaStreamSynchronize (s));
  return shift_plan_check (P);
}

} /* namespace lgh */

using namespace lgh;

/* ======================================================================== */

extern "C" {

lgh_glr_opts_t
lgh_glr_opts_default (void)
{
  /* glr_common_impl.h:295-312 */
  lgh_glr_opts_t o;
  o.ell = 200;
  o.q_power = 1;
  o.trunc_abs = 0.;
  o.trunc_rel = 1e-3;
  o.treat = LGH_TREAT_FLIP;
  o.seed = 271828UL;
  o.backend = LGH_GLR_DEFAULT;
  o.nb = 64;
  o.panel = 64;
  o.grid2d = 0;
  o.check = 1;
  return o;
}

lgh_exec_opts_t
lgh_exec_opts_default (void)
{
  lgh_exec_opts_t e;
  e.precision = LGH_PREC_FP64;
  e.inner_rtol = 0.;
  e.verbose = 0;
  e.rank_cap = 0;
  e.check_form = LGH_CHECK_PROJ;
  return e;
}

/* the communicator of the lgh_glr_compute_cols call on this thread */
static thread_local const lgh_comm_t *t_comm = nullptr;

int
lgh_glr_compute_ex (lgh_Mat B, lgh_prior_t *prior, const lgh_glr_opts_t *opts,
                    const lgh_exec_opts_t *exec, lgh_glr_t **glr,
                    lgh_glr_report_t *report)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (B && prior && glr, LGH_ERR_ARG_NULL, "lgh_glr_compute: NULL argument");
  LGH_CHECK (B->kind == 0, LGH_ERR_ARG_WRONG, "lgh_glr_compute: B must be a CSR Mat");
  /* row slabs: B and the prior's Z sharded by the same communicator */
  const bool rows = B->rows != nullptr || prior->rows != nullptr;
  if (rows) {
    LGH_CHECK (B->rows && prior->rows, LGH_ERR_ARG_WRONG,
               "lgh_glr_compute: B and the prior must both be row-sharded "
               "or neither");
    LGH_CHECK (rows_same_comm (B->rows->comm, prior->Z->rows->comm)
               && B->rows->N == prior->Z->rows->N
               && B->rows->row0 == prior->Z->rows->row0
               && B->rows->row1 == prior->Z->rows->row1, LGH_ERR_ARG_WRONG,
               "lgh_glr_compute: B and the prior are sharded differently");
    LGH_CHECK (t_comm == nullptr, LGH_ERR_SUP,
               "lgh_glr_compute: row slabs and column sharding together");
  }
  LGH_CHECK (B->csr.n == prior->n, LGH_ERR_ARG_SIZ, "lgh_glr_compute: B and prior sizes differ");
  const int64_t Nglob = rows ? B->rows->N : B->csr.n;
  lgh_glr_opts_t o = opts ? *opts : lgh_glr_opts_default ();
  /* glr_common_impl.h:651-654 */
  LGH_CHECK (o.ell > 0 && o.ell <= Nglob, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_compute: need 0 < ell (%d) <= N (%d)", o.ell, (int) Nglob);
  LGH_CHECK (o.ell <= 2048, LGH_ERR_SUP, "lgh_glr_compute: ell %d > 2048 on one device", o.ell);
  LGH_CHECK (o.treat >= 0 && o.treat <= 2, LGH_ERR_ARG_OUTOFRANGE, "lgh_glr_compute: treat");
  lgh_glr_t *g = new lgh_glr_t ();
  g->n = B->csr.n;
  g->opts = o;
  g->exec = exec ? *exec : lgh_exec_opts_default ();
  LGH_CHECK (g->exec.precision == LGH_PREC_FP64 || g->exec.precision == LGH_PREC_MIXED,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_glr_compute: precision");
  g->B = B;
  B->refs++;
  g->prior = prior;
  prior_ref (prior);
  if (t_comm) g->comm = *t_comm;
  g->N = Nglob;
  if (rows) {
    g->rows = &B->rows->comm;
    g->row0 = B->rows->row0;
  }
  lgh_glr_report_t rep;
  int rc = (g->exec.precision == LGH_PREC_MIXED) ? build<float> (g, &rep)
                                                 : build<double> (g, &rep);
  if (rc) {
    lgh_glr_destroy (g);
    return rc;
  }
  if (report) *report = rep;
  *glr = g;
  return 0;
}

int
lgh_glr_compute (lgh_Mat B, lgh_prior_t *prior, const lgh_glr_opts_t *opts,
                 lgh_glr_t **glr, lgh_glr_report_t *report)
{
  return lgh_glr_compute_ex (B, prior, opts, nullptr, glr, report);
}

void
lgh_cols_range (int w, int rank, int size, int *c0, int *c1)
{
  const int groups = (w + 3) / 4;
  const int g0 = (int) ((int64_t) groups * rank / size);
  const int g1 = (int) ((int64_t) groups * (rank + 1) / size);
  *c0 = std::min (w, 4 * g0);
  *c1 = std::min (w, 4 * g1);
}

size_t
lgh_cols_exchange_bytes (int64_t n, int ell, int size)
{
  int wmax = 0, c0, c1;
  for (int r = 0; r < size; r++) {
    lgh_cols_range (ell, r, size, &c0, &c1);
    wmax = std::max (wmax, c1 - c0);
  }
  return (size_t) n * round_ld (std::max (wmax, 1)) * sizeof (double);
}

int
lgh_glr_compute_cols (lgh_Mat B, lgh_prior_t *prior, const lgh_glr_opts_t *opts,
                      const lgh_exec_opts_t *exec, const lgh_comm_t *comm,
                      lgh_glr_t **glr, lgh_glr_report_t *report)
{
  LGH_CHECK (comm && comm->allgather && comm->size >= 1 && comm->rank >= 0
             && comm->rank < comm->size, LGH_ERR_ARG_WRONG,
             "lgh_glr_compute_cols: need a communicator with 0 <= rank < size "
             "and an all-gather");
  t_comm = comm;
  const int rc = lgh_glr_compute_ex (B, prior, opts, exec, glr, report);
  t_comm = nullptr;
  return rc;
}

int
lgh_glr_extend (lgh_glr_t *glr, int k_new, lgh_glr_report_t *report)
{
  /* glr_common_impl.h:684-719 */
  LGH_CHECK (glr, LGH_ERR_ARG_NULL, "lgh_glr_extend: NULL");
  LGH_CHECK (!glr->corrected, LGH_ERR_ORDER,
             "lgh_glr_extend: not available after lgh_glr_correct");
  LGH_CHECK (k_new > 0, LGH_ERR_ARG_OUTOFRANGE, "lgh_glr_extend: k_new must be positive");
  LGH_CHECK (glr->opts.ell + k_new <= glr->n, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_glr_extend: extended ell (%d) exceeds N (%d)",
             glr->opts.ell + k_new, (int) glr->n);
  LGH_CHECK (glr->opts.ell + k_new <= 2048, LGH_ERR_SUP, "lgh_glr_extend: ell > 2048");
  lgh_glr_report_t rep;
  const int mixed = glr->exec.precision == LGH_PREC_MIXED;
  int rc;
  if (glr->opts.backend == LGH_GLR_REPLICATED) {
    /* replicated backend: recompute at the wider ell (:711-715) */
    glr->opts.ell += k_new;
    rc = mixed ? build<float> (glr, &rep) : build<double> (glr, &rep);
  } else {
    rc = mixed ? extend_incremental<float> (glr, k_new, &rep)
               : extend_incremental<double> (glr, k_new, &rep);
  }
  if (rc) return rc;
  if (report) *report = rep;
  return 0;
}

void
lgh_glr_destroy (lgh_glr_t *glr)
{
  if (glr == NULL) return;
  shift_plan_free (glr->splan);
  glr->splan = nullptr;
  if (glr->B) mat_release (glr->B);
  lgh_prior_destroy (glr->prior);
  delete glr;
}

int
lgh_glr_batch_info (const lgh_glr_t *glr, long *graph_captures,
                    long *graph_replays, int *tile_variant, int *tuned_shapes)
{
  LGH_CHECK (glr, LGH_ERR_ARG_NULL, "lgh_glr_batch_info: NULL");
  long c = 0, r = 0;
  int v = -1;
  shift_plan_stats (glr->splan, &c, &r, &v);
  if (graph_captures) *graph_captures = c;
  if (graph_replays) *graph_replays = r;
  if (tile_variant) *tile_variant = v;
  if (tuned_shapes) *tuned_shapes = tune_table_size ();
  return 0;
}

int
lgh_glr_solve (lgh_glr_t *glr, double c, lgh_Vec rhs, lgh_Vec x)
{
  /* H(c)^{-1} = Z^{-T} M^{1/2} (F + cI)^{-1} M^{1/2} Z^{-1}
   * (glr_common_impl.h:1007-1024) */
  LGH_TRY (check_vecs (glr, rhs, x, "lgh_glr_solve"));
  LGH_TRY (check_shift (glr, c, "lgh_glr_solve"));
  LGH_TRY (glr_scratch (glr));
  lgh_prior_t *p = glr->prior;
  LGH_TRY (prior_solve_vec (p, rhs->d, nullptr, glr->w1.p, p->msqrt.p));
  LGH_TRY (filter_core (glr, 0, c, 0., nullptr, 1. / c, glr->w1.p, glr->w2.p));
  LGH_TRY (prior_solve_vec (p, glr->w2.p, p->msqrt.p, x->d, nullptr));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  return 0;
}

int
lgh_glr_apply (lgh_glr_t *glr, double c, lgh_Vec v, lgh_Vec y)
{
  /* exact y = B v + c R v (glr_common_impl.h:1026-1048); after a
   * correction the corrected low-rank action (correct.cu) */
  LGH_TRY (check_vecs (glr, v, y, "lgh_glr_apply"));
  if (glr->corrected) return glr_apply_corrected (glr, c, v->d, y->d);
  LGH_TRY (glr_scratch (glr));
  lgh_prior_t *p = glr->prior;
  cudaStream_t s = stream ();
  LGH_TRY (mat_mult_vec (glr->B, v->d, y->d));
  LGH_TRY (prior_applyZ (p, v->d, glr->w1.p));
  LGH_TRY (launch_vec_div (glr->n, glr->w1.p, p->mass.p, glr->w2.p, s));
  LGH_TRY (prior_applyZ (p, glr->w2.p, glr->w1.p));
  LGH_TRY (launch_vec_axpby (glr->n, 1.0, y->d, c, glr->w1.p, y->d, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

int
lgh_glr_factor (lgh_glr_t *glr, double c, lgh_factor_t which, lgh_Vec in,
                lgh_Vec out)
{
  /* G = Z M^{-1/2} S, S = (F + cI)^{1/2} (glr_common_impl.h:1050-1097) */
  LGH_TRY (check_vecs (glr, in, out, "lgh_glr_factor"));
  LGH_TRY (check_shift (glr, c, "lgh_glr_factor"));
  LGH_TRY (glr_scratch (glr));
  lgh_prior_t *p = glr->prior;
  cudaStream_t s = stream ();
  switch (which) {
  case LGH_FACTOR_G:
    LGH_TRY (filter_core (glr, 2, c, 0., nullptr, sqrt (c), in->d, glr->w1.p));
    LGH_TRY (launch_vec_scale (glr->n, glr->w1.p, p->minvsqrt.p, 1.0, glr->w2.p, s));
    LGH_TRY (prior_applyZ (p, glr->w2.p, out->d));
    break;
  case LGH_FACTOR_GT:
    LGH_TRY (prior_applyZ (p, in->d, glr->w1.p));
    LGH_TRY (launch_vec_scale (glr->n, glr->w1.p, p->minvsqrt.p, 1.0, glr->w2.p, s));
    LGH_TRY (filter_core (glr, 2, c, 0., nullptr, sqrt (c), glr->w2.p, out->d));
    break;
  case LGH_FACTOR_GINV:
    LGH_TRY (prior_solve_vec (p, in->d, nullptr, glr->w1.p, p->msqrt.p));
    LGH_TRY (filter_core (glr, 1, c, 0., nullptr, 1. / sqrt (c), glr->w1.p, out->d));
    break;
  case LGH_FACTOR_GINVT:
    LGH_TRY (filter_core (glr, 1, c, 0., nullptr, 1. / sqrt (c), in->d, glr->w1.p));
    LGH_TRY (prior_solve_vec (p, glr->w1.p, p->msqrt.p, out->d, nullptr));
    break;
  default:
    return set_error (LGH_ERR_ARG_OUTOFRANGE, "lgh_glr_factor: unknown factor action");
  }
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

int
lgh_glr_sample (lgh_glr_t *glr, double c, lgh_Vec xi, lgh_Vec x)
{
  /* x = G^{-T} xi (glr_common_impl.h:1099-1104) */
  return lgh_glr_factor (glr, c, LGH_FACTOR_GINVT, xi, x);
}

double
lgh_glr_logdet (lgh_glr_t *glr, double c)
{
  /* glr_common_impl.h:988-997: no floor check; returns the value */
  if (glr == NULL || glr->kept == 0) return 0.;
  double out = 0.;
  lgh_glr_logdet_batch (glr, 1, &c, &out);
  return out;
}

int
lgh_glr_logdet_batch (lgh_glr_t *glr, int nshift, const double *c, double *out)
{
  LGH_CHECK (glr && c && out, LGH_ERR_ARG_NULL, "lgh_glr_logdet_batch: NULL");
  LGH_CHECK (nshift > 0, LGH_ERR_ARG_SIZ, "lgh_glr_logdet_batch: nshift");
  if (glr->kept == 0) {
    for (int i = 0; i < nshift; i++) out[i] = 0.;
    return 0;
  }
  cudaStream_t s = stream ();
  DBuf<double> cd, od;
  LGH_TRY (cd.alloc (nshift));
  LGH_TRY (od.alloc (nshift));
  LGH_CUDA (cudaMemcpyAsync (cd.p, c, nshift * sizeof (double), cudaMemcpyHostToDevice, s));
  k_logdet<<<nshift, 256, 0, s>>> (glr->kept, glr->lam_d.p, nshift, cd.p, od.p);
  LGH_LAUNCH_CHECK ();
  LGH_CUDA (cudaMemcpyAsync (out, od.p, nshift * sizeof (double), cudaMemcpyDeviceToHost, s));
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

int
lgh_glr_pow (lgh_glr_t *glr, double c, double p, lgh_Vec in, lgh_Vec out)
{
  /* glr_common_impl.h:975-986 */
  LGH_TRY (check_vecs (glr, in, out, "lgh_glr_pow"));
  LGH_TRY (check_shift (glr, c, "lgh_glr_pow"));
  LGH_TRY (filter_core (glr, 3, c, p, nullptr, pow (c, p), in->d, out->d));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  return 0;
}

int
lgh_glr_filter (lgh_glr_t *glr, const double *f_lam, double f_c, lgh_Vec in,
                lgh_Vec out)
{
  /* glr_common_impl.h:968-973 */
  LGH_TRY (check_vecs (glr, in, out, "lgh_glr_filter"));
  LGH_CHECK (f_lam || glr->kept == 0, LGH_ERR_ARG_NULL, "lgh_glr_filter: f_lam NULL");
  LGH_TRY (filter_core (glr, 5, 0., 0., f_lam, f_c, in->d, out->d));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  return 0;
}

int
lgh_glr_eigs (const lgh_glr_t *glr, int *nkept, const double **lam)
{
  /* glr_common_impl.h:999-1005: borrowed, valid until extend/destroy */
  LGH_CHECK (glr && nkept && lam, LGH_ERR_ARG_NULL, "lgh_glr_eigs: NULL");
  *nkept = glr->kept;
  *lam = glr->lam_h.data ();
  return 0;
}

int
lgh_glr_get_stats (const lgh_glr_t *glr, lgh_glr_stats_t *st)
{
  LGH_CHECK (glr && st, LGH_ERR_ARG_NULL, "lgh_glr_get_stats: NULL");
  *st = glr->stats;
  st->n = glr->n;
  st->ell = glr->opts.ell;
  st->kept = glr->kept;
  st->precision = glr->exec.precision;
  const lgh::ZsolveStats &z = glr->prior->stats;
  st->zsolve_calls = z.calls;
  st->zsolve_iters = z.block_iters;
  st->zsolve_mean_col_iters = z.cols ? (double) z.col_iters / z.cols : 0.;
  st->device_bytes = (int64_t) (glr->U.n + glr->Q.n + glr->A.n + glr->Wz.n) * 8
                     + (int64_t) (glr->U32.n + glr->Q32.n) * 4;
  return 0;
}

int
lgh_glr_get_U (const lgh_glr_t *glr, double *U_dev, int64_t ld)
{
  LGH_CHECK (glr && U_dev, LGH_ERR_ARG_NULL, "lgh_glr_get_U: NULL");
  LGH_CHECK (ld >= glr->n, LGH_ERR_ARG_SIZ, "lgh_glr_get_U: ld");
  if (glr->kept == 0) return 0;
  LGH_TRY (launch_rowmajor_to_colmajor (glr->n, glr->kept, glr->U.p, glr->ldu,
                                        U_dev, ld, nullptr, stream ()));
  LGH_CUDA (cudaStreamSynchronize (stream ()));
  return 0;
}

int
lgh_glr_solve_batch (lgh_glr_t *glr, int nshift, const double *c, int m,
                     const double *rhs, int64_t ldr, double *x, int64_t ldx)
{
  LGH_CHECK (glr, LGH_ERR_ARG_NULL, "lgh_glr_solve_batch: NULL");
  return batch_op (glr, 0, nshift, c, m, rhs, ldr, x, ldx);
}

int
lgh_glr_sample_batch (lgh_glr_t *glr, int nshift, const double *c, int m,
                      const double *xi, int64_t ldr, double *x, int64_t ldx)
{
  LGH_CHECK (glr, LGH_ERR_ARG_NULL, "lgh_glr_sample_batch: NULL");
  return batch_op (glr, 1, nshift, c, m, xi, ldr, x, ldx);
}

} /* extern "C" */
