/* batch.cu -- many shifts x many right-hand sides: the shift-combination
 * stage of lgh_glr_solve_batch / lgh_glr_sample_batch as one captured
 * launch sequence.
 *
 * The batched operations write, for every shift c and right-hand side r,
 *   solve:  x_c = (1/c) y0 + W diag(1/(lam + c) - 1/c) U^T r2
 *   sample: x_c = c^(-1/2) y0 + W diag((lam + c)^(-1/2) - c^(-1/2)) U^T xi
 * with the shift-independent W = Z^{-1} M^{1/2} U and y0, r2 (the
 * reference's per-call lgh_glr_solve / lgh_glr_sample, glr_common_impl.h:
 * 1007-1024 and 1084-1104, with the Z-solves hoisted out of the shift
 * loop).  After the shift-independent Z-solves, the rest is a fixed-shape
 * sequence: upload the call's output pointer and shifts from a pinned
 * parameter block, tabulate the per-shift coefficients, and one fused
 * GEMM over all shifts (k_shift_combine) that writes the caller's
 * column-major output.  A ShiftPlan keeps the workspace of one object and
 * the sequence captured as a CUDA graph; a call whose kind, shift count
 * and width match the captured ones only refreshes the pinned block and
 * replays the graph.  Tile shape of the combination: chosen per shape by
 * the autotuner (tune.cu).
 */

#include <string.h>

#include <algorithm>

#include "lgh_batch.h"
#include "lgh_internal.h"
#include "lgh_objects.h"

namespace lgh
{

namespace
{

/* g[k + si kept] = f(lam_k + c_si) - f(c_si), fc[si] = f(c_si);
 * f(x) = 1/x (solve) or x^(-1/2) (sample) */
__global__ void
k_shift_table (int kept, int nshift, const double *__restrict__ lam,
               const double *__restrict__ c, int kind, double *__restrict__ g,
               double *__restrict__ fc)
{
  const int64_t total = (int64_t) kept * nshift;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int si = (int) (e / kept);
    const int k = (int) (e - (int64_t) si * kept);
    const double cs = c[si];
    const double f0 = kind == 0 ? 1. / cs : 1. / sqrt (cs);
    const double x = lam[k] + cs;
    g[e] = (kind == 0 ? 1. / x : 1. / sqrt (x)) - f0;
    if (k == 0) fc[si] = f0;
  }
  if (kept == 0)
    for (int si = blockIdx.x * blockDim.x + threadIdx.x; si < nshift;
         si += gridDim.x * blockDim.x)
      fc[si] = kind == 0 ? 1. / c[si] : 1. / sqrt (c[si]);
}

/* the pinned per-call parameters: output pointer and leading dimension */
struct Params
{
  double *out;
  int64_t ldo;
};

} /* namespace */

struct ShiftPlan
{
  int64_t n = 0;
  int m = 0, kept = 0, cap_shift = 0;
  /* workspace of the batched operation (stable addresses for the graph) */
  DBuf<double> R, Xs, Y0, Wc, work, g, fc, cdev;
  DBuf<char> pdev;
  Params *ph = nullptr;   /* pinned */
  double *cph = nullptr;  /* pinned shifts */
  /* the captured sequence and what it was captured for */
  cudaStream_t cs = nullptr;
  /* one captured tail per kind (0 solve, 1 sample) and what it was
   * captured for */
  struct Captured
  {
    cudaGraphExec_t exec = nullptr;
    int nshift = 0, m = 0, variant = -1;
    const double *W = nullptr, *lam = nullptr;
  } cap[2];
  long replays = 0, captures = 0;
  int last_variant = -1;
  /* the tensor-core form (mixed-precision objects): W split once, the
   * coefficient block split per call, tensor maps of both tile widths */
  int kpad = 0, ncolp = 0;
  DBuf<float> Ah, Al, Bh, Bl;
  DBuf<int> err;
  const double *a_W = nullptr;
  int a_kept = -1;
  UmmaMaps maps[2];
  bool maps_ok = false;

  ~ShiftPlan ()
  {
    drop_graph ();
    if (cs) cudaStreamDestroy (cs);
    if (ph) cudaFreeHost (ph);
    if (cph) cudaFreeHost (cph);
  }

  void drop_graph ()
  {
    for (auto &c : cap) {
      if (c.exec) cudaGraphExecDestroy (c.exec);
      c = Captured ();
    }
  }

  int ensure (int64_t n_, int m_, int kept_, int nshift)
  {
    if (n_ != n || m_ > m || kept_ != kept) {
      drop_graph ();
      n = n_;
      m = std::max (m, m_);
      kept = kept_;
      const int ld = round_ld (m);
      LGH_TRY (R.alloc ((size_t) n * ld));
      LGH_TRY (Xs.alloc ((size_t) n * ld));
      LGH_TRY (Y0.alloc ((size_t) n * ld));
      LGH_TRY (Wc.alloc ((size_t) std::max (kept, 1) * m));
      LGH_TRY (work.alloc (std::max<size_t> (gemm_tn_work_elems (n, std::max (kept, 1), m), 64)));
    }
    if (nshift > cap_shift) {
      drop_graph ();
      cap_shift = std::max (nshift, 64);
      LGH_TRY (g.alloc ((size_t) std::max (kept, 1) * cap_shift));
      LGH_TRY (fc.alloc (cap_shift));
      LGH_TRY (cdev.alloc (cap_shift));
      if (cph) cudaFreeHost (cph);
      cph = nullptr;
      LGH_CUDA (cudaMallocHost ((void **) &cph, cap_shift * sizeof (double)));
    }
    if (!ph) {
      LGH_CUDA (cudaMallocHost ((void **) &ph, sizeof (Params)));
      LGH_TRY (pdev.alloc (sizeof (Params)));
    }
    if (!cs) LGH_CUDA (cudaStreamCreateWithFlags (&cs, cudaStreamNonBlocking));
    return 0;
  }
};

/* the tensor-core operands of a mixed-precision object: A from W (when
 * W or kept changed), B's buffers for nshift x m columns, the tensor maps */
int
shift_plan_prepare_umma (ShiftPlan *P, lgh_glr_t *g, int nshift, int m)
{
  cudaStream_t s = stream ();
  const int kpad = std::max (32, (P->kept + 31) / 32 * 32);
  const int ncolp = (nshift * m + 255) / 256 * 256;
  bool remap = false;
  if (!P->err.p) {
    LGH_TRY (P->err.alloc (1));
    LGH_CUDA (cudaMemsetAsync (P->err.p, 0, sizeof (int), s));
  }
  if (kpad != P->kpad || P->a_W != g->Wz.p || P->a_kept != P->kept) {
    P->drop_graph ();
    P->kpad = kpad;
    LGH_TRY (P->Ah.alloc ((size_t) P->n * kpad));
    LGH_TRY (P->Al.alloc ((size_t) P->n * kpad));
    LGH_TRY (umma_split_rows (P->n, P->kept, kpad, g->Wz.p, g->ldu, P->Ah.p,
                              P->Al.p, s));
    P->a_W = g->Wz.p;
    P->a_kept = P->kept;
    remap = true;
  }
  if (ncolp > P->ncolp) {
    P->drop_graph ();
    P->ncolp = ncolp;
    LGH_TRY (P->Bh.alloc ((size_t) ncolp * kpad));
    LGH_TRY (P->Bl.alloc ((size_t) ncolp * kpad));
    remap = true;
  }
  if (remap || !P->maps_ok) {
    P->maps_ok = false;
    LGH_TRY (umma_encode (&P->maps[0], P->Ah.p, P->Al.p, P->n, P->Bh.p, P->Bl.p,
                          P->ncolp, P->kpad, 128));
    LGH_TRY (umma_encode (&P->maps[1], P->Ah.p, P->Al.p, P->n, P->Bh.p, P->Bl.p,
                          P->ncolp, P->kpad, 256));
    P->maps_ok = true;
  }
  return 0;
}

/* a failed pipeline wait in the tensor-core kernel since the last check */
int
shift_plan_check (ShiftPlan *P)
{
  if (!P->err.p) return 0;
  int e = 0;
  LGH_CUDA (cudaMemcpy (&e, P->err.p, sizeof (int), cudaMemcpyDeviceToHost));
  if (e) {
    LGH_CUDA (cudaMemset (P->err.p, 0, sizeof (int)));
    return set_error (LGH_ERR_GPU, "batched combination: a tensor-core "
                      "pipeline wait ran out (code %d)", e);
  }
  return 0;
}

/* the fixed-shape tail: parameters up, coefficient table, combination */
static int
enqueue_tail (ShiftPlan &P, lgh_glr_t *g, int kind, int nshift, int variant,
              int m, cudaStream_t s)
{
  Params *pd = (Params *) P.pdev.p;
  LGH_CUDA (cudaMemcpyAsync (pd, P.ph, sizeof (Params), cudaMemcpyHostToDevice, s));
  LGH_CUDA (cudaMemcpyAsync (P.cdev.p, P.cph, nshift * sizeof (double),
                             cudaMemcpyHostToDevice, s));
  const int64_t tot = std::max<int64_t> ((int64_t) P.kept * nshift, nshift);
  const int grid = (int) std::min<int64_t> ((tot + 255) / 256, 1024);
  k_shift_table<<<std::max (grid, 1), 256, 0, s>>> (P.kept, nshift, g->lam_d.p,
                                                    P.cdev.p, kind, P.g.p, P.fc.p);
  LGH_LAUNCH_CHECK ();
  if (variant >= kShiftVariants) {
    LGH_CHECK (P.maps_ok, LGH_ERR_ARG_WRONGSTATE, "batch: tensor maps missing");
    LGH_TRY (umma_split_coef (P.kept, P.kpad, m, nshift, P.ncolp, P.g.p, P.Wc.p,
                              P.Bh.p, P.Bl.p, s));
    const int u = variant - kShiftVariants;
    return launch_shift_combine_umma (P.maps[u & 1], umma_variant_stages (u),
                                      P.n, P.kpad, m, nshift, P.fc.p, P.Y0.p,
                                      round_ld (m), &pd->out, &pd->ldo,
                                      P.err.p, s);
  }
  return launch_shift_combine_variant (variant, P.n, P.kept, m, nshift, g->Wz.p,
                                       g->ldu, P.Wc.p, P.g.p, P.fc.p, P.Y0.p,
                                       round_ld (m), &pd->out, &pd->ldo, s);
}

int
shift_plan_get (lgh_glr_t *g, int64_t n, int m, int kept, int nshift,
                ShiftPlan **out)
{
  if (!g->splan) g->splan = new ShiftPlan ();
  LGH_TRY (g->splan->ensure (n, m, kept, nshift));
  *out = g->splan;
  return 0;
}

double *shift_plan_R (ShiftPlan *P) { return P->R.p; }
double *shift_plan_Xs (ShiftPlan *P) { return P->Xs.p; }
double *shift_plan_Y0 (ShiftPlan *P) { return P->Y0.p; }
double *shift_plan_Wc (ShiftPlan *P) { return P->Wc.p; }
double *shift_plan_work (ShiftPlan *P, size_t *elems)
{
  *elems = P->work.n;
  return P->work.p;
}

/* run the tail for one call: the pinned block gets the call's output and
 * shifts; the graph is (re)captured when the kind, shift count, width,
 * tile variant or W changed, then replayed on the library's stream */
int
shift_plan_combine (ShiftPlan *P, lgh_glr_t *g, int kind, int nshift,
                    const double *c_host, int m, double *x, int64_t ldx,
                    int variant)
{
  cudaStream_t s = stream ();
  /* the previous replay has completed (every call synchronises), so the
   * pinned block is free to rewrite */
  P->ph->out = x;
  P->ph->ldo = ldx;
  memcpy (P->cph, c_host, nshift * sizeof (double));
  ShiftPlan::Captured &C = P->cap[kind & 1];
  if (C.exec == nullptr || C.nshift != nshift || C.m != m
      || C.variant != variant || C.W != g->Wz.p || C.lam != g->lam_d.p) {
    if (C.exec) cudaGraphExecDestroy (C.exec);
    C = ShiftPlan::Captured ();
    /* captured on the plan's own stream; the instantiated graph is then
     * launched on the library's stream, after the work queued there */
    cudaGraph_t gr = nullptr;
    int rc = 0;
    if (cudaStreamBeginCapture (P->cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      rc = enqueue_tail (*P, g, kind, nshift, variant, m, P->cs);
      const cudaError_t ce = cudaStreamEndCapture (P->cs, &gr);
      if (!rc && (ce != cudaSuccess || gr == nullptr
                  || cudaGraphInstantiate (&C.exec, gr, 0) != cudaSuccess)) {
        C.exec = nullptr;
      }
      if (gr) cudaGraphDestroy (gr);
    }
    cudaGetLastError ();
    if (rc) return rc;
    if (C.exec) {
      C.nshift = nshift;
      C.m = m;
      C.variant = variant;
      C.W = g->Wz.p;
      C.lam = g->lam_d.p;
      P->captures++;
    }
  }
  P->last_variant = variant;
  if (C.exec) {
    LGH_CUDA (cudaGraphLaunch (C.exec, s));
    P->replays++;
  } else {
    /* capture unavailable: the same sequence, eagerly */
    LGH_TRY (enqueue_tail (*P, g, kind, nshift, variant, m, s));
  }
  return 0;
}

/* the same sequence run eagerly on the library's stream (the autotuner's
 * trials, timed without capture overhead) */
int
shift_plan_run_eager (ShiftPlan *P, lgh_glr_t *g, int kind, int nshift,
                      const double *c_host, int m, double *x, int64_t ldx,
                      int variant)
{
  cudaStream_t s = stream ();
  LGH_CUDA (cudaStreamSynchronize (s));   /* the pinned block is free */
  P->ph->out = x;
  P->ph->ldo = ldx;
  memcpy (P->cph, c_host, nshift * sizeof (double));
  LGH_TRY (enqueue_tail (*P, g, kind, nshift, variant, m, s));
  P->last_variant = variant;
  return 0;
}

void
shift_plan_stats (const ShiftPlan *P, long *captures, long *replays,
                  int *last_variant)
{
  *captures = P ? P->captures : 0;
  *replays = P ? P->replays : 0;
  *last_variant = P ? P->last_variant : -1;
}

void
shift_plan_free (ShiftPlan *P)
{
  delete P;
}

} /* namespace lgh */
