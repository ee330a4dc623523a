/* server.cu -- the request loop: continuous batching of solve / sample /
 * logdet requests on a resident GLR object.
 *
 * A worker thread owns a fixed-width block of PCG "slots" (columns of the
 * blocked Z-solve).  Every column carries its own CG scalars and
 * convergence mask, so columns at different iteration counts share one
 * tick (p-update + Z product + x/r update + preconditioner + dots); a
 * converged column is harvested at the next check and its slot is refilled
 * with the next stage of its request or with a newly admitted request.
 * Work of requests that arrive while others are on the GPU therefore joins
 * the same launches, and one column's arithmetic never depends on the
 * other columns (the same request gives the same bits alone or in a mix).
 *
 * Stages (the shift-independent form of glr_common_impl.h:1007-1024 and
 * 1084-1091 with W = Z^{-1} M^{1/2} U precomputed once):
 *   solve  (m columns, shift c): y1 = Z^{-1} r; r2 = M^{1/2} y1;
 *          w = U^T r2; y0 = Z^{-1} (M^{1/2} r2);
 *          x = (1/c) y0 + W diag(1/(lam+c) - 1/c) w
 *   sample (m columns, shift c): w = U^T xi; y0 = Z^{-1} (M^{1/2} xi);
 *          x = c^{-1/2} y0 + W diag((lam+c)^{-1/2} - c^{-1/2}) w
 *   logdet (shift c): sum log(lam + c) - log c, at admission.
 * Admission: a request waits until enough slots are free for all of its
 * columns and the device has room for its staging buffers plus a reserve.
 */

#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "lgh_device.cuh"
#include "lgh_internal.h"
#include "lgh_mg.h"
#include "lgh_objects.h"

namespace lgh
{

/* kernels of zsolve.cu used by the tick (declared there) */
template <typename T>
int server_tick_pq (const Csr &Z, const T *Zb, const T *Pold, T *Pnew, T *Q,
                    int ld, ZWork &ws, cudaStream_t s);
template <typename T>
int server_tick_upd (int64_t n, int ld, T *X, T *R, const T *Pn, const T *Q,
                     ZWork &ws, cudaStream_t s);
template <typename T>
int server_tick_dots (const Csr &Z, const T *R, const T *Zb, int ld, int w,
                      const int *fresh, double rtol, ZWork &ws, cudaStream_t s);

/* column copy between a contiguous device column and a strided column of
 * a row-major block, with an optional row scale */
__global__ void
k_col_in (int64_t n, const double *src, const double *scale, double *blk,
          int ld, int col)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    blk[i * ld + col] = scale ? scale[i] * src[i] : src[i];
}

__global__ void
k_col_out (int64_t n, const double *blk, int ld, int col, const double *scale,
           double *dst)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    dst[i] = scale ? scale[i] * blk[i * ld + col] : blk[i * ld + col];
}

__global__ void
k_col_zero (int64_t n, double *blk, int ld, int col)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x)
    blk[i * ld + col] = 0.;
}

/* D[k] = (f(lam_k + c) - f(c)) w[k] for one column; kind 0 solve, 1 sample */
__global__ void
k_coef_col (int kept, const double *lam, double c, int kind, const double *w,
            double *d)
{
  const double fc = (kind == 0) ? 1. / c : 1. / sqrt (c);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < kept;
       k += gridDim.x * blockDim.x) {
    const double x = lam[k] + c;
    const double f = (kind == 0) ? 1. / x : 1. / sqrt (x);
    d[k] = (f - fc) * w[k];
  }
}

__global__ void
k_logdet1 (int kept, const double *lam, double c, double *out)
{
  __shared__ double red[256];
  double s = 0.;
  const double lc = log (c);
  for (int i = threadIdx.x; i < kept; i += blockDim.x) s += log (lam[i] + c) - lc;
  red[threadIdx.x] = s;
  __syncthreads ();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads ();
  }
  if (threadIdx.x == 0) *out = red[0];
}

static int
cgrid (int64_t n)
{
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > num_sms () * 8) g = num_sms () * 8;
  return (int) g;
}

struct SReq
{
  int64_t id = 0;
  int kind = 0;
  double c = 1.;
  int m = 0;
  const double *hin = nullptr;
  int64_t ldin = 0;
  double *hout = nullptr;
  int64_t ldout = 0;
  /* device staging: input columns, output columns, U^T coefficients */
  DBuf<double> din, dout, wcoef;
  int cols_left = 0;
  int status = 1;   /* 1 pending/active, 0 done, < 0 error */
  double t_submit = 0., t_done = 0.;
  std::vector<int> stage;   /* per column */
};

struct Slot
{
  SReq *req = nullptr;
  int col = -1;
  int stage = 0;  /* 1: first Z-solve, 2: second (solve only) */
};

} /* namespace lgh */

struct lgh_server
{
  lgh_glr_t *g = nullptr;
  int cap = 64, ld = 64;
  double reserve = 0.1;
  cudaStream_t s = nullptr;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<lgh::SReq *> pending;
  std::map<int64_t, std::unique_ptr<lgh::SReq>> reqs;
  std::atomic<bool> stop{ false };
  int64_t next_id = 1;
  int err = 0;
  std::string errmsg;
  /* slot block */
  lgh::ZWork ws;
  lgh::DBuf<double> Pold_extra;
  std::vector<lgh::Slot> slots;
  lgh::DBuf<int> fresh_d;
  std::vector<int> fresh_h;
  lgh::DBuf<double> colbuf, coefbuf, gemmwork;
  /* statistics */
  long completed = 0, ticks = 0, cols_done = 0;
  std::vector<double> lat;
  double t0 = 0., t_last = 0.;
};

namespace lgh
{

static int
srv_fail (lgh_server_t *sv, int rc)
{
  std::lock_guard<std::mutex> lk (sv->mu);
  sv->err = rc;
  sv->errmsg = lgh_last_error ();
  for (auto &kv : sv->reqs)
    if (kv.second->status == 1) kv.second->status = -rc;
  sv->done_cv.notify_all ();
  return rc;
}

/* admit as many pending requests as slots and memory allow (host side) */
static int
srv_admit (lgh_server_t *sv, std::vector<SReq *> &admitted)
{
  std::lock_guard<std::mutex> lk (sv->mu);
  int free_slots = 0;
  for (auto &sl : sv->slots) free_slots += sl.req == nullptr;
  while (!sv->pending.empty ()) {
    SReq *r = sv->pending.front ();
    if (r->kind != 2 && r->m > free_slots) break;
    size_t fb = 0, tb = 0;
    cudaMemGetInfo (&fb, &tb);
    const double need = (double) sv->g->n * r->m * 16 + (double) sv->g->kept * r->m * 8;
    if ((double) fb - need < sv->reserve * (double) tb && r->kind != 2) break;
    sv->pending.pop_front ();
    admitted.push_back (r);
    if (r->kind != 2) free_slots -= r->m;
  }
  return 0;
}

/* write a column into slot `sl`: R = rhs, X = 0, next-Pold = 0, fresh */
static int
srv_place (lgh_server_t *sv, int sl, const double *rhs, const double *scale,
           double *Pnext)
{
  const int64_t n = sv->g->n;
  double *X = (double *) sv->ws.X.p, *R = (double *) sv->ws.R.p;
  k_col_in<<<cgrid (n), 256, 0, sv->s>>> (n, rhs, scale, R, sv->ld, sl);
  k_col_zero<<<cgrid (n), 256, 0, sv->s>>> (n, X, sv->ld, sl);
  k_col_zero<<<cgrid (n), 256, 0, sv->s>>> (n, Pnext, sv->ld, sl);
  LGH_LAUNCH_CHECK ();
  sv->fresh_h[sl] = 1;
  return 0;
}

static void
srv_loop (lgh_server_t *sv)
{
  lgh_glr_t *g = sv->g;
  lgh_prior_t *p = g->prior;
  const int64_t n = g->n;
  const int ld = sv->ld;
  cudaStream_t s = sv->s;
  double *X = (double *) sv->ws.X.p, *R = (double *) sv->ws.R.p;
  double *P0 = (double *) sv->ws.P0.p, *P1 = (double *) sv->ws.P1.p;
  double *Q = (double *) sv->ws.Q.p, *Zb = (double *) sv->ws.Zb.p;
  double *Pold = P0, *Pnew = P1;
  const double *ms = p->msqrt.p, *mass = p->mass.p;
  const int kept = g->kept;
  int rc = 0;
  cudaMemsetAsync (P0, 0, (size_t) n * ld * 8, s);
  cudaMemsetAsync (P1, 0, (size_t) n * ld * 8, s);
  cudaMemsetAsync (R, 0, (size_t) n * ld * 8, s);
  cudaMemsetAsync (X, 0, (size_t) n * ld * 8, s);
  cudaMemsetAsync (sv->ws.ival.p, 0, sv->ws.ival.n * sizeof (int), s);
  cudaStreamSynchronize (s);
  while (!sv->stop.load ()) {
    /* 1. admission of new requests into free slots */
    std::vector<SReq *> adm;
    srv_admit (sv, adm);
    for (SReq *r : adm) {
      if (r->kind == 2) {
        /* logdet at admission */
        DBuf<double> cd;
        double *dv = nullptr;
        rc = cd.alloc (1);
        if (!rc && kept > 0) {
          dv = cd.p;
          k_logdet1<<<1, 256, 0, s>>> (kept, g->lam_d.p, r->c, dv);
        }
        double hv = 0.;
        if (!rc && kept > 0 && cudaMemcpyAsync (&hv, dv, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess)
          rc = set_error (LGH_ERR_GPU, "server: logdet copy");
        if (!rc) cudaStreamSynchronize (s);
        std::lock_guard<std::mutex> lk (sv->mu);
        if (r->hout) *r->hout = hv;
        r->status = rc ? -rc : 0;
        r->t_done = wall ();
        sv->lat.push_back (r->t_done - r->t_submit);
        sv->completed++;
        sv->done_cv.notify_all ();
        continue;
      }
      /* stage the input columns and (sample) the U^T coefficients */
      rc = r->din.alloc ((size_t) n * r->m);
      if (!rc) rc = r->dout.alloc ((size_t) n * r->m);
      if (!rc) rc = r->wcoef.alloc ((size_t) std::max (kept, 1) * r->m);
      if (!rc) {
        for (int j = 0; j < r->m; j++)
          if (cudaMemcpyAsync (r->din.p + (size_t) j * n, r->hin + (size_t) j * r->ldin,
                               n * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = set_error (LGH_ERR_GPU, "server: input copy");
      }
      if (!rc && r->kind == 1 && kept > 0)
        rc = launch_gemm_tn<double> (n, kept, r->m, g->U.p, g->ldu, r->din.p, 1,
                                     r->wcoef.p, kept, 0, sv->gemmwork.p,
                                     sv->gemmwork.n, s);
      r->stage.assign (r->m, 1);
      r->cols_left = r->m;
      int j = 0;
      for (int sl = 0; sl < sv->cap && j < r->m && !rc; sl++) {
        if (sv->slots[sl].req) continue;
        sv->slots[sl].req = r;
        sv->slots[sl].col = j;
        sv->slots[sl].stage = 1;
        /* solve: stage-1 rhs r; sample: M^{1/2} xi */
        rc = srv_place (sv, sl, r->din.p + (size_t) j * n,
                        r->kind == 1 ? ms : nullptr, Pold);
        j++;
      }
      if (rc) break;
    }
    if (rc) { srv_fail (sv, rc); return; }
    bool any = false;
    for (auto &sl : sv->slots) any |= sl.req != nullptr;
    if (!any) {
      std::unique_lock<std::mutex> lk (sv->mu);
      sv->cv.wait_for (lk, std::chrono::milliseconds (2),
                       [&] { return sv->stop.load () || !sv->pending.empty (); });
      continue;
    }
    /* 2. one tick: Z = PC(R) for fresh columns happens inside the tick order
     *    pq -> upd -> PC -> dots; fresh columns were placed before PC */
    rc = cudaMemcpyAsync (sv->fresh_d.p, sv->fresh_h.data (), sv->cap * sizeof (int),
                          cudaMemcpyHostToDevice, s) == cudaSuccess ? 0
         : set_error (LGH_ERR_GPU, "server: fresh flags");
    if (!rc) {
      if (p->mg) rc = mg_vcycle<double> (p->mg, R, Zb, ld, sv->cap, s);
      else rc = launch_rowscale<double> (n, ld, p->Z->csr.dinv, R, ld, Zb, ld, s);
    }
    if (!rc) rc = server_tick_dots<double> (p->Z->csr, R, Zb, ld, sv->cap,
                                            sv->fresh_d.p, p->zcfg.rtol, sv->ws, s);
    std::fill (sv->fresh_h.begin (), sv->fresh_h.end (), 0);
    if (!rc) rc = server_tick_pq<double> (p->Z->csr, Zb, Pold, Pnew, Q, ld, sv->ws, s);
    if (!rc) rc = server_tick_upd<double> (n, ld, X, R, Pnew, Q, sv->ws, s);
    std::swap (Pold, Pnew);
    sv->ticks++;
    /* 3. harvest converged columns */
    std::vector<int> act (sv->cap);
    if (!rc && cudaMemcpyAsync (act.data (), sv->ws.ival.p, sv->cap * sizeof (int),
                                cudaMemcpyDeviceToHost, s) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "server: mask copy");
    if (!rc && cudaStreamSynchronize (s) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "server: tick");
    if (rc) { srv_fail (sv, rc); return; }
    for (int sl = 0; sl < sv->cap && !rc; sl++) {
      Slot &S = sv->slots[sl];
      if (!S.req || act[sl] || sv->fresh_h[sl]) continue;
      SReq *r = S.req;
      const int j = S.col;
      double *ycol = r->dout.p + (size_t) j * n;
      if (r->kind == 0 && S.stage == 1) {
        /* y1 -> r2 = M^{1/2} y1 (kept in dout), w = U^T r2, stage-2 rhs M y1 */
        k_col_out<<<cgrid (n), 256, 0, s>>> (n, X, ld, sl, ms, ycol);
        if (kept > 0)
          rc = launch_gemm_tn<double> (n, kept, 1, g->U.p, g->ldu, ycol, 1,
                                       r->wcoef.p + (size_t) j * kept, kept, 0,
                                       sv->gemmwork.p, sv->gemmwork.n, s);
        if (!rc) {
          /* the stage-2 right-hand side M^{1/2} r2 */
          k_col_out<<<cgrid (n), 256, 0, s>>> (n, X, ld, sl, mass, sv->colbuf.p);
          rc = srv_place (sv, sl, sv->colbuf.p, nullptr, Pold);
          S.stage = 2;
        }
        continue;
      }
      /* final stage: y0 in X; x = a y0 + W diag(f - f_c) w */
      const double a = (r->kind == 0) ? 1. / r->c : 1. / sqrt (r->c);
      k_col_out<<<cgrid (n), 256, 0, s>>> (n, X, ld, sl, nullptr, sv->colbuf.p);
      if (kept > 0) {
        k_coef_col<<<1, 256, 0, s>>> (kept, g->lam_d.p, r->c, r->kind,
                                      r->wcoef.p + (size_t) j * kept, sv->coefbuf.p);
        rc = launch_gemm_nn<double> (n, kept, 1, 1.0, g->Wz.p, g->ldu,
                                     sv->coefbuf.p, kept, a, sv->colbuf.p, 1,
                                     ycol, 1, s);
      } else {
        rc = launch_vec_scale (n, sv->colbuf.p, nullptr, a, ycol, s);
      }
      if (rc) break;
      if (cudaMemcpyAsync (r->hout + (size_t) j * r->ldout, ycol, n * 8,
                           cudaMemcpyDeviceToHost, s) != cudaSuccess) {
        rc = set_error (LGH_ERR_GPU, "server: output copy");
        break;
      }
      S.req = nullptr;
      S.col = -1;
      S.stage = 0;
      r->cols_left--;
      sv->cols_done++;
      if (r->cols_left == 0) {
        if (cudaStreamSynchronize (s) != cudaSuccess) {
          rc = set_error (LGH_ERR_GPU, "server: completion");
          break;
        }
        std::lock_guard<std::mutex> lk (sv->mu);
        r->status = 0;
        r->t_done = wall ();
        sv->lat.push_back (r->t_done - r->t_submit);
        sv->completed++;
        sv->t_last = r->t_done;
        r->din.release ();
        r->dout.release ();
        r->wcoef.release ();
        sv->done_cv.notify_all ();
      }
    }
    if (rc) { srv_fail (sv, rc); return; }
  }
}

} /* namespace lgh */

using namespace lgh;

extern "C" {

lgh_server_opts_t
lgh_server_opts_default (void)
{
  lgh_server_opts_t o;
  o.slots = 64;
  o.hbm_reserve = 0.05;
  o.verbose = 0;
  return o;
}

int
lgh_server_create (lgh_glr_t *glr, const lgh_server_opts_t *opts,
                   lgh_server_t **out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (glr && out, LGH_ERR_ARG_NULL, "lgh_server_create: NULL");
  LGH_CHECK (glr->prior->is_mat, LGH_ERR_SUP,
             "lgh_server_create: needs a Mat-path prior (device Z-solves)");
  lgh_server_opts_t o = opts ? *opts : lgh_server_opts_default ();
  LGH_CHECK (o.slots >= 1 && o.slots <= 512, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_server_create: slots %d", o.slots);
  lgh_server_t *sv = new lgh_server_t ();
  sv->g = glr;
  sv->cap = o.slots;
  sv->ld = round_ld (o.slots);
  sv->reserve = o.hbm_reserve;
  int rc = 0;
  if (cudaStreamCreateWithFlags (&sv->s, cudaStreamNonBlocking) != cudaSuccess)
    rc = set_error (LGH_ERR_GPU, "lgh_server_create: stream");
  /* the shift-independent precompute W = Z^{-1} M^{1/2} U */
  if (!rc && glr->kept > 0 && !glr->have_wz) {
    rc = glr->Wz.alloc ((size_t) glr->n * glr->ldu);
    if (!rc) cudaMemset (glr->Wz.p, 0, (size_t) glr->n * glr->ldu * 8);
    if (!rc) rc = prior_solve_rows<double> (glr->prior, glr->kept, glr->U.p,
                                            glr->ldu, glr->prior->msqrt.p,
                                            glr->Wz.p, glr->ldu, nullptr);
    if (!rc) glr->have_wz = 1;
  }
  if (!rc) rc = sv->ws.alloc (glr->n, sv->ld, 0);
  if (!rc) rc = sv->fresh_d.alloc (sv->ld);
  if (!rc) rc = sv->colbuf.alloc (glr->n);
  if (!rc) rc = sv->coefbuf.alloc (std::max (glr->kept, 1));
  if (!rc) rc = sv->gemmwork.alloc (std::max<size_t> (
             gemm_tn_work_elems (glr->n, std::max (glr->kept, 1), sv->cap), 64));
  if (rc) {
    if (sv->s) cudaStreamDestroy (sv->s);
    delete sv;
    return rc;
  }
  sv->slots.assign (sv->cap, Slot ());
  sv->fresh_h.assign (sv->ld, 0);
  sv->t0 = wall ();
  int dev = 0;
  cudaGetDevice (&dev);
  sv->worker = std::thread ([sv, dev] {
    cudaSetDevice (dev);
    srv_loop (sv);
  });
  *out = sv;
  return 0;
}

int
lgh_server_submit (lgh_server_t *sv, int kind, double c, int m,
                   const double *in, int64_t ldin, double *out, int64_t ldout,
                   int64_t *id)
{
  LGH_CHECK (sv && id, LGH_ERR_ARG_NULL, "lgh_server_submit: NULL");
  LGH_CHECK (kind >= 0 && kind <= 2, LGH_ERR_ARG_OUTOFRANGE, "lgh_server_submit: kind");
  LGH_CHECK (c > sv->g->floor, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_server_submit: shift c must exceed the spectrum floor %g",
             sv->g->floor);
  if (kind != 2) {
    LGH_CHECK (in && out && m >= 1 && m <= sv->cap && ldin >= sv->g->n
               && ldout >= sv->g->n, LGH_ERR_ARG_SIZ,
               "lgh_server_submit: need 1 <= m <= slots and ld >= n");
  }
  std::unique_ptr<SReq> r (new SReq ());
  r->kind = kind;
  r->c = c;
  r->m = kind == 2 ? 0 : m;
  r->hin = in;
  r->ldin = ldin;
  r->hout = out;
  r->ldout = ldout;
  r->t_submit = wall ();
  std::lock_guard<std::mutex> lk (sv->mu);
  LGH_CHECK (sv->err == 0, sv->err, "lgh_server_submit: server failed: %s",
             sv->errmsg.c_str ());
  r->id = sv->next_id++;
  *id = r->id;
  sv->pending.push_back (r.get ());
  sv->reqs[r->id] = std::move (r);
  sv->cv.notify_all ();
  return 0;
}

int
lgh_server_wait (lgh_server_t *sv, int64_t id, double timeout_s, double *latency_s)
{
  LGH_CHECK (sv, LGH_ERR_ARG_NULL, "lgh_server_wait: NULL");
  std::unique_lock<std::mutex> lk (sv->mu);
  auto it = sv->reqs.find (id);
  LGH_CHECK (it != sv->reqs.end (), LGH_ERR_ARG_WRONG, "lgh_server_wait: unknown id");
  SReq *r = it->second.get ();
  const bool ok = sv->done_cv.wait_for (
      lk, std::chrono::duration<double> (timeout_s), [&] { return r->status != 1; });
  if (!ok) return set_error (LGH_ERR_NOT_CONVERGED, "lgh_server_wait: timed out");
  if (r->status < 0) return set_error (-r->status, "lgh_server_wait: %s", sv->errmsg.c_str ());
  if (latency_s) *latency_s = r->t_done - r->t_submit;
  sv->reqs.erase (it);
  return 0;
}

int
lgh_server_get_stats (lgh_server_t *sv, lgh_server_stats_t *st)
{
  LGH_CHECK (sv && st, LGH_ERR_ARG_NULL, "lgh_server_get_stats: NULL");
  std::lock_guard<std::mutex> lk (sv->mu);
  std::vector<double> l = sv->lat;
  std::sort (l.begin (), l.end ());
  memset (st, 0, sizeof (*st));
  st->completed = sv->completed;
  st->columns = sv->cols_done;
  st->ticks = sv->ticks;
  st->pending = (long) sv->pending.size ();
  if (!l.empty ()) {
    st->p50_s = l[l.size () / 2];
    st->p99_s = l[std::min (l.size () - 1, (size_t) (0.99 * l.size ()))];
    st->max_s = l.back ();
  }
  const double el = (sv->t_last > sv->t0) ? sv->t_last - sv->t0 : 0.;
  st->columns_per_s = el > 0. ? sv->cols_done / el : 0.;
  return 0;
}

void
lgh_server_destroy (lgh_server_t *sv)
{
  if (!sv) return;
  sv->stop.store (true);
  sv->cv.notify_all ();
  if (sv->worker.joinable ()) sv->worker.join ();
  if (sv->s) cudaStreamDestroy (sv->s);
  delete sv;
}

} /* extern "C" */
