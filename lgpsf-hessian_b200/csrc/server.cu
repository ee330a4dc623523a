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
 * The loop has its own stream, Z-solve workspace and V-cycle level
 * buffers; it only reads the GLR object (U, lambda, W) and the prior's
 * operators, so other read-only calls may run beside it.
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

int ensure_wz (lgh_glr_t *g);
int launch_logdet (int kept, const double *lam, int nshift, const double *c,
                   double *out, cudaStream_t s);

/* a contiguous device column into column `col` of a row-major block, with
 * an optional row scale; the same column of X and of the next direction
 * block are cleared (a fresh CG start) */
__global__ void
k_col_place (int64_t n, const double *src, const double *scale, double *R,
             double *X, double *P, int ld, int col)
{
  for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t) gridDim.x * blockDim.x) {
    R[i * ld + col] = scale ? scale[i] * src[i] : src[i];
    X[i * ld + col] = 0.;
    P[i * ld + col] = 0.;
  }
}

/* H[i, t] = colscale[t] * rowscale[i] * X[i, slot[t]] (rowscale nullable) */
__global__ void
k_gather_slots (int64_t n, const double *__restrict__ X, int ld,
                const int *__restrict__ slot, const double *__restrict__ colscale,
                const double *__restrict__ rowscale, int k, double *H, int ldh)
{
  const int64_t total = n * k;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / k;
    const int t = (int) (e - i * k);
    double v = colscale[t] * X[i * ld + slot[t]];
    if (rowscale) v *= rowscale[i];
    H[i * ldh + t] = v;
  }
}

/* second Z-solve of a solve request, in place: R = mass * X, X = 0, P = 0 */
__global__ void
k_restage (int64_t n, double *X, double *R, double *P, int ld,
           const int *__restrict__ slot, int k, const double *__restrict__ mass)
{
  const int64_t total = n * k;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / k;
    const int64_t o = i * ld + slot[(int) (e - i * k)];
    R[o] = mass[i] * X[o];
    X[o] = 0.;
    P[o] = 0.;
  }
}

/* dst[t][i] = H[i, t] */
__global__ void
k_scatter_cols (int64_t n, const double *__restrict__ H, int ldh, int k,
                double *const *dst)
{
  const int64_t total = n * k;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int t = (int) (e / n);
    const int64_t i = e - (int64_t) t * n;
    dst[t][i] = H[i * ldh + t];
  }
}

/* coefficient columns kept x k: D[:, t] = (f(lam + c_t) - f(c_t)) w_t with
 * f = 1/x (solve) or x^{-1/2} (sample); the same arithmetic as the batched
 * operations' shift coefficients */
__global__ void
k_coef_cols (int kept, const double *__restrict__ lam, int k,
             const double *__restrict__ c, const int *__restrict__ kind,
             const double *const *w, double *D)
{
  const int64_t total = (int64_t) kept * k;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int t = (int) (e / kept);
    const int j = (int) (e - (int64_t) t * kept);
    const double cs = c[t], x = lam[j] + cs;
    const double f = kind[t] == 0 ? 1. / x - 1. / cs : 1. / sqrt (x) - 1. / sqrt (cs);
    D[e] = f * w[t][j];
  }
}

/* wdst[t][0..kept) = C[:, t] */
__global__ void
k_put_coef (int kept, int k, const double *__restrict__ C, double *const *wdst)
{
  const int64_t total = (int64_t) kept * k;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int t = (int) (e / kept);
    wdst[t][e - (int64_t) t * kept] = C[e];
  }
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
  int staged = 0;     /* din holds the input (set by the copier)          */
  int placed = 0;     /* columns handed to slots so far                   */
  int cols_left = 0;  /* columns not yet through their last stage         */
  cudaEvent_t ev_out = nullptr;   /* recorded after the last scatter      */
  int status = 1;     /* 1 pending/active, 0 done, < 0 error              */
  double t_submit = 0., t_done = 0.;
  double t_staged = 0., t_placed = 0., t_ran = 0.;   /* stage timestamps */
};

struct Slot
{
  SReq *req = nullptr;
  int col = -1;
  int stage = 0;  /* 1: first Z-solve, 2: second (solve only) */
};

/* per-harvest description of the harvested columns, copied to the device */
struct Harvest
{
  static constexpr int MAXS = 512;
  int slot_a[MAXS];          /* solve columns leaving stage 1 */
  int slot_b[MAXS];          /* columns leaving their last stage */
  int kind_b[MAXS];
  double one[MAXS];
  double scale_b[MAXS];      /* 1/c (solve) or c^{-1/2} (sample) */
  double c_b[MAXS];
  double *wdst_a[MAXS];      /* request coefficient columns */
  const double *wsrc_b[MAXS];
  double *out_b[MAXS];       /* request output columns */
};

/* a run of one request's columns admitted into slots in one admission pass */
struct Adm
{
  SReq *r;
  int j0, take;
};

} /* namespace lgh */

struct lgh_server
{
  lgh_glr_t *g = nullptr;
  int cap = 64, ld = 64;
  int pc32 = 0;                 /* FP32 V-cycle (mixed-precision object) */
  double reserve = 0.1;
  cudaStream_t s = nullptr;     /* the loop's stream */
  cudaStream_t sc = nullptr;    /* the copier's stream */
  std::thread worker, copier;
  std::mutex mu;
  std::condition_variable cv, ccv, done_cv;
  std::deque<lgh::SReq *> pending;      /* arrival order, until placed */
  std::deque<lgh::SReq *> up_q, dl_q;   /* copier: inputs in, results out */
  std::map<int64_t, std::unique_ptr<lgh::SReq>> reqs;
  std::atomic<bool> stop{ false };
  std::atomic<int> failed{ 0 };
  int64_t next_id = 1;
  long staged_cols = 0;   /* uploaded columns not yet placed */
  long inflight = 0;      /* requests holding device staging */
  int err = 0;
  std::string errmsg;
  /* slot block and per-tick staging */
  lgh::ZWork ws;
  std::vector<lgh::MgWork> mgw;   /* own V-cycle level buffers */
  std::vector<lgh::Slot> slots;
  lgh::DBuf<int> fresh_d;
  std::vector<int> fresh_h;
  int *fresh_pin = nullptr, *act_pin = nullptr;   /* pinned per-tick copies */
  /* the copier's pinned staging, two halves of stg_half bytes: host
   * columns are packed into one half by memcpy while the other half's
   * DMA runs, so no pageable copy (which the driver stages itself,
   * holding up other threads' calls) is ever made */
  char *stg = nullptr;
  size_t stg_half = 0;
  cudaEvent_t stg_ev[2] = { nullptr, nullptr };
  lgh::DBuf<double> H, coef, gemmwork, ldc, ldo;
  lgh::DBuf<char> hv_d;
  std::unique_ptr<lgh::Harvest> hv;
  /* statistics */
  long completed = 0;
  std::atomic<long> ticks{ 0 }, cols_done{ 0 }, harvests{ 0 };   /* loop-written */
  double t_admit = 0., t_tick = 0., t_harvest = 0., t_up = 0., t_down = 0.;
  double occ_sum = 0.;                 /* occupied slots summed over ticks */
  double st_stage = 0., st_admit = 0., st_run = 0., st_out = 0.;
  long st_n = 0;                       /* solve / sample requests timed   */
  std::vector<double> lat;
  double t0 = 0., t_last = 0.;
};

namespace lgh
{

static int
srv_fail (lgh_server_t *sv, int rc)
{
  std::lock_guard<std::mutex> lk (sv->mu);
  if (sv->err == 0) {
    sv->err = rc;
    sv->errmsg = lgh_last_error ();
  }
  sv->failed.store (rc);
  for (auto &kv : sv->reqs)
    if (kv.second->status == 1) kv.second->status = -rc;
  sv->cv.notify_all ();
  sv->ccv.notify_all ();
  sv->done_cv.notify_all ();
  return rc;
}

/* a request leaves the loop: its staging is released (every use of it on
 * either stream has completed: the copier synchronised its stream after
 * the result copy, which waited for the loop's last scatter) */
static void
srv_finish (lgh_server_t *sv, SReq *r, int rc)
{
  const bool held = r->din.p != nullptr;
  r->din.release ();
  r->dout.release ();
  r->wcoef.release ();
  if (r->ev_out) {
    cudaEventDestroy (r->ev_out);
    r->ev_out = nullptr;
  }
  std::lock_guard<std::mutex> lk (sv->mu);
  r->status = rc ? -rc : 0;
  r->t_done = wall ();
  if (held) sv->inflight--;
  if (!rc) {
    sv->lat.push_back (r->t_done - r->t_submit);
    sv->completed++;
    sv->t_last = r->t_done;
    if (r->kind != 2) {
      sv->st_stage += r->t_staged - r->t_submit;
      sv->st_admit += r->t_placed - r->t_staged;
      sv->st_run += r->t_ran - r->t_placed;
      sv->st_out += r->t_done - r->t_ran;
      sv->st_n++;
    }
  }
  sv->done_cv.notify_all ();
  sv->ccv.notify_all ();
}

/* room on the device for a request's staging above the reserve; the
 * allocation cache's free blocks count as free (blocks that objects built
 * before this loop released stay cached, and the driver does not see
 * them as free) */
static bool
srv_room (lgh_server_t *sv, const SReq *r)
{
  size_t fb = 0, tb = 0;
  if (cudaMemGetInfo (&fb, &tb) != cudaSuccess) {
    cudaGetLastError ();
    return true;
  }
  const double avail = (double) fb + (double) pool_cached_bytes ();
  const double need = (double) sv->g->n * r->m * 16.
                      + (double) std::max (sv->g->kept, 1) * r->m * 8.;
  return avail - need >= sv->reserve * (double) tb;
}

/* a request's input columns to the device through the pinned halves */
static int
srv_put (lgh_server_t *sv, SReq *r)
{
  const int64_t n = sv->g->n;
  const size_t colb = (size_t) n * 8;
  const int per = (int) std::max<size_t> (1, sv->stg_half / colb);
  int b = 0;
  for (int j0 = 0; j0 < r->m; j0 += per, b ^= 1) {
    const int mc = std::min (per, r->m - j0);
    char *h = sv->stg + (size_t) b * sv->stg_half;
    LGH_CUDA (cudaEventSynchronize (sv->stg_ev[b]));   /* the half is free */
    /* host memory bandwidth takes several threads */
#pragma omp parallel for num_threads (std::min (mc, 8)) schedule (static)
    for (int j = 0; j < mc; j++)
      memcpy (h + (size_t) j * colb, r->hin + (size_t) (j0 + j) * r->ldin, colb);
    LGH_CUDA (cudaMemcpyAsync (r->din.p + (size_t) j0 * n, h, mc * colb,
                               cudaMemcpyHostToDevice, sv->sc));
    LGH_CUDA (cudaEventRecord (sv->stg_ev[b], sv->sc));
  }
  LGH_CUDA (cudaStreamSynchronize (sv->sc));
  return 0;
}

/* a finished request's output columns to the host through the pinned
 * halves: chunk k + 1's DMA runs while chunk k is copied out */
static int
srv_get (lgh_server_t *sv, SReq *r)
{
  const int64_t n = sv->g->n;
  const size_t colb = (size_t) n * 8;
  const int per = (int) std::max<size_t> (1, sv->stg_half / colb);
  const int nch = (r->m + per - 1) / per;
  LGH_CUDA (cudaStreamWaitEvent (sv->sc, r->ev_out, 0));
  auto issue = [&] (int k) -> int {
    const int b = k & 1, j0 = k * per, mc = std::min (per, r->m - j0);
    LGH_CUDA (cudaMemcpyAsync (sv->stg + (size_t) b * sv->stg_half,
                               r->dout.p + (size_t) j0 * n, mc * colb,
                               cudaMemcpyDeviceToHost, sv->sc));
    LGH_CUDA (cudaEventRecord (sv->stg_ev[b], sv->sc));
    return 0;
  };
  LGH_TRY (issue (0));
  for (int k = 0; k < nch; k++) {
    if (k + 1 < nch) LGH_TRY (issue (k + 1));
    const int b = k & 1, j0 = k * per, mc = std::min (per, r->m - j0);
    LGH_CUDA (cudaEventSynchronize (sv->stg_ev[b]));
    const char *h = sv->stg + (size_t) b * sv->stg_half;
#pragma omp parallel for num_threads (std::min (mc, 8)) schedule (static)
    for (int j = 0; j < mc; j++)
      memcpy (r->hout + (size_t) (j0 + j) * r->ldout, h + (size_t) j * colb, colb);
  }
  return 0;
}

/* the copier thread: host transfers off the loop's critical path.  Inputs
 * go up in arrival order, at most two slot blocks of columns ahead of
 * placement and while the device keeps hbm_reserve free (or nothing else
 * holds staging); results come down as soon as the loop's last scatter
 * of a request has run, and the request completes when they have landed. */
static void
srv_copier (lgh_server_t *sv)
{
  const int64_t n = sv->g->n;
  const long ahead = 2L * sv->cap;
  for (;;) {
    SReq *dl = nullptr, *up = nullptr;
    bool room_wait = false;
    {
      std::unique_lock<std::mutex> lk (sv->mu);
      auto may_up = [&] {
        return !sv->up_q.empty ()
               && (sv->staged_cols == 0
                   || sv->staged_cols + sv->up_q.front ()->m <= ahead);
      };
      sv->ccv.wait_for (lk, std::chrono::milliseconds (5), [&] {
        return sv->stop.load () || sv->failed.load () || !sv->dl_q.empty ()
               || may_up ();
      });
      if (sv->stop.load () || sv->failed.load ()) return;
      if (!sv->dl_q.empty ()) {
        dl = sv->dl_q.front ();
        sv->dl_q.pop_front ();
      } else if (may_up ()) {
        SReq *r = sv->up_q.front ();
        if (r->status != 1) {
          sv->up_q.pop_front ();
        } else if (sv->inflight > 0 && !srv_room (sv, r)) {
          room_wait = true;
        } else {
          sv->up_q.pop_front ();
          up = r;
        }
      }
    }
    if (room_wait) {
      std::this_thread::sleep_for (std::chrono::milliseconds (1));
      continue;
    }
    if (dl) {
      const double w0 = wall ();
      const int rc = srv_get (sv, dl);
      {
        std::lock_guard<std::mutex> lk (sv->mu);
        sv->t_down += wall () - w0;
      }
      srv_finish (sv, dl, rc);
      if (rc) { srv_fail (sv, rc); return; }
    } else if (up) {
      /* all of the request's device staging, so that the loop thread
       * never allocates */
      int rc = up->din.alloc ((size_t) n * up->m);
      if (!rc) rc = up->dout.alloc ((size_t) n * up->m);
      if (!rc) rc = up->wcoef.alloc ((size_t) std::max (sv->g->kept, 1) * up->m);
      if (rc == 0) {
        std::lock_guard<std::mutex> lk (sv->mu);
        sv->inflight++;
      }
      if (rc == LGH_ERR_MEM) {
        /* this request alone fails: nothing else held staging memory */
        up->din.release ();
        up->dout.release ();
        up->wcoef.release ();
        srv_finish (sv, up, rc);
        clear_error ();
        continue;
      }
      const double w0 = wall ();
      if (!rc) rc = srv_put (sv, up);
      if (rc) { srv_fail (sv, rc); return; }
      std::lock_guard<std::mutex> lk (sv->mu);
      sv->t_up += wall () - w0;
      up->t_staged = wall ();
      up->staged = 1;
      sv->staged_cols += up->m;
      sv->cv.notify_all ();
    }
  }
}

/* admit staged requests in arrival order, column by column, into the free
 * slots: a request wider than what is free starts with the columns that
 * fit and keeps the head of the queue until all of its columns are in */
static void
srv_admit (lgh_server_t *sv, std::vector<Adm> &adm)
{
  std::lock_guard<std::mutex> lk (sv->mu);
  int free_slots = 0;
  for (auto &sl : sv->slots) free_slots += sl.req == nullptr;
  while (!sv->pending.empty ()) {
    SReq *r = sv->pending.front ();
    if (r->status != 1) {           /* failed while staging */
      sv->pending.pop_front ();
      continue;
    }
    if (!r->staged) break;
    if (r->kind == 2) {
      sv->pending.pop_front ();
      adm.push_back ({ r, 0, 0 });
      continue;
    }
    const int take = std::min (free_slots, r->m - r->placed);
    if (take <= 0) break;
    adm.push_back ({ r, r->placed, take });
    r->placed += take;
    free_slots -= take;
    if (r->placed == r->m) {
      sv->pending.pop_front ();
      sv->staged_cols -= r->m;
      sv->ccv.notify_all ();
    }
  }
}

/* logdet requests complete at admission with the kernel of lgh_glr_logdet */
static int
srv_logdet (lgh_server_t *sv, SReq *r)
{
  lgh_glr_t *g = sv->g;
  double v = 0.;
  if (g->kept > 0) {
    LGH_CUDA (cudaMemcpyAsync (sv->ldc.p, &r->c, 8, cudaMemcpyHostToDevice, sv->s));
    LGH_TRY (launch_logdet (g->kept, g->lam_d.p, 1, sv->ldc.p, sv->ldo.p, sv->s));
    LGH_CUDA (cudaMemcpyAsync (&v, sv->ldo.p, 8, cudaMemcpyDeviceToHost, sv->s));
    LGH_CUDA (cudaStreamSynchronize (sv->s));
  }
  if (r->hout) *r->hout = v;
  srv_finish (sv, r, 0);
  return 0;
}

/* columns j0 .. j0 + take - 1 of a solve / sample request into free slots;
 * its first run also forms, for a sample, w = U^T xi for all of its
 * columns (the copier allocated the request's staging) */
static int
srv_start (lgh_server_t *sv, const Adm &a, double *Pold)
{
  lgh_glr_t *g = sv->g;
  SReq *r = a.r;
  const int64_t n = g->n;
  const int kept = g->kept, ldh = sv->ld;
  cudaStream_t s = sv->s;
  double *X = (double *) sv->ws.X.p, *R = (double *) sv->ws.R.p;
  if (a.j0 == 0) {
    r->cols_left = r->m;
    r->t_placed = wall ();
    if (r->kind == 1 && kept > 0) {
      for (int c0 = 0; c0 < r->m; c0 += sv->cap) {
        const int mc = std::min (sv->cap, r->m - c0);
        LGH_TRY (launch_colmajor_to_rowmajor (n, mc, r->din.p + (size_t) c0 * n, n,
                                              sv->H.p, ldh, nullptr, s));
        LGH_TRY (launch_gemm_tn<double> (n, kept, mc, g->U.p, g->ldu, sv->H.p, ldh,
                                         r->wcoef.p + (size_t) c0 * kept, kept, 0,
                                         sv->gemmwork.p, sv->gemmwork.n, s));
      }
    }
  }
  int j = a.j0;
  const int jend = a.j0 + a.take;
  for (int sl = 0; sl < sv->cap && j < jend; sl++) {
    Slot &S = sv->slots[sl];
    if (S.req) continue;
    S.req = r;
    S.col = j;
    S.stage = 1;
    /* first right-hand side: r (solve) or M^{1/2} xi (sample) */
    k_col_place<<<cgrid (n), 256, 0, s>>> (n, r->din.p + (size_t) j * n,
                                           r->kind == 1 ? g->prior->msqrt.p : nullptr,
                                           R, X, Pold, sv->ld, sl);
    LGH_LAUNCH_CHECK ();
    sv->fresh_h[sl] = 1;
    j++;
  }
  LGH_CHECK (j == jend, LGH_ERR_ARG_WRONG, "server: admitted without free slots");
  return 0;
}

/* columns whose Z-solve has converged move on: solve stage 1 -> U^T
 * coefficients and the second Z-solve; last stage -> the Woodbury
 * combination and the output column.  A request whose last column left
 * goes to the copier behind an event on the loop's stream. */
static int
srv_harvest (lgh_server_t *sv, const std::vector<int> &act, double *Pold)
{
  lgh_glr_t *g = sv->g;
  const int64_t n = g->n;
  const int kept = g->kept, ld = sv->ld, ldh = sv->ld;
  cudaStream_t s = sv->s;
  double *X = (double *) sv->ws.X.p, *R = (double *) sv->ws.R.p;
  Harvest &h = *sv->hv;
  int ka = 0, kb = 0;
  std::vector<SReq *> fin;
  for (int sl = 0; sl < sv->cap; sl++) {
    Slot &S = sv->slots[sl];
    if (!S.req || act[sl] || sv->fresh_h[sl]) continue;
    SReq *r = S.req;
    if (r->kind == 0 && S.stage == 1) {
      h.slot_a[ka] = sl;
      h.one[ka] = 1.;
      h.wdst_a[ka] = r->wcoef.p + (size_t) S.col * std::max (kept, 1);
      ka++;
      S.stage = 2;
      sv->fresh_h[sl] = 1;
    } else {
      h.slot_b[kb] = sl;
      h.kind_b[kb] = r->kind;
      h.c_b[kb] = r->c;
      h.scale_b[kb] = r->kind == 0 ? 1. / r->c : 1. / sqrt (r->c);
      h.wsrc_b[kb] = r->wcoef.p + (size_t) S.col * std::max (kept, 1);
      h.out_b[kb] = r->dout.p + (size_t) S.col * n;
      kb++;
      S.req = nullptr;
      S.col = -1;
      S.stage = 0;
      if (--r->cols_left == 0) fin.push_back (r);
    }
  }
  if (ka == 0 && kb == 0) return 0;
  sv->harvests++;
  Harvest *hd = (Harvest *) sv->hv_d.p;
  LGH_CUDA (cudaMemcpyAsync (hd, &h, sizeof (Harvest), cudaMemcpyHostToDevice, s));
  if (ka > 0) {
    /* r2 = M^{1/2} y1 -> w = U^T r2; then the second right-hand side M y1 */
    if (kept > 0) {
      k_gather_slots<<<cgrid (n * ka), 256, 0, s>>> (n, X, ld, hd->slot_a, hd->one,
                                                     g->prior->msqrt.p, ka, sv->H.p, ldh);
      LGH_LAUNCH_CHECK ();
      LGH_TRY (launch_gemm_tn<double> (n, kept, ka, g->U.p, g->ldu, sv->H.p, ldh,
                                       sv->coef.p, kept, 0, sv->gemmwork.p,
                                       sv->gemmwork.n, s));
      k_put_coef<<<cgrid ((int64_t) kept * ka), 256, 0, s>>> (kept, ka, sv->coef.p,
                                                              hd->wdst_a);
      LGH_LAUNCH_CHECK ();
    }
    k_restage<<<cgrid (n * ka), 256, 0, s>>> (n, X, R, Pold, ld, hd->slot_a, ka,
                                              g->prior->mass.p);
    LGH_LAUNCH_CHECK ();
  }
  if (kb > 0) {
    /* x = a y0 + W diag(f(lam + c) - f(c)) w */
    k_gather_slots<<<cgrid (n * kb), 256, 0, s>>> (n, X, ld, hd->slot_b, hd->scale_b,
                                                   nullptr, kb, sv->H.p, ldh);
    LGH_LAUNCH_CHECK ();
    if (kept > 0) {
      k_coef_cols<<<cgrid ((int64_t) kept * kb), 256, 0, s>>> (kept, g->lam_d.p, kb,
                                                               hd->c_b, hd->kind_b,
                                                               hd->wsrc_b, sv->coef.p);
      LGH_LAUNCH_CHECK ();
      LGH_TRY (launch_gemm_nn<double> (n, kept, kb, 1.0, g->Wz.p, g->ldu, sv->coef.p,
                                       kept, 1.0, sv->H.p, ldh, sv->H.p, ldh, s));
    }
    k_scatter_cols<<<cgrid (n * kb), 256, 0, s>>> (n, sv->H.p, ldh, kb, hd->out_b);
    LGH_LAUNCH_CHECK ();
    sv->cols_done += kb;
  }
  const double tr = wall ();
  for (SReq *r : fin) {
    r->t_ran = tr;
    LGH_CUDA (cudaEventCreateWithFlags (&r->ev_out, cudaEventDisableTiming));
    LGH_CUDA (cudaEventRecord (r->ev_out, s));
  }
  if (!fin.empty ()) {
    std::lock_guard<std::mutex> lk (sv->mu);
    for (SReq *r : fin) sv->dl_q.push_back (r);
    sv->ccv.notify_all ();
  }
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
  float *R32 = (float *) sv->ws.R32.p, *Z32 = (float *) sv->ws.Z32.p;
  double *Pold = P0, *Pnew = P1;
  int rc = 0;
  const size_t blk = (size_t) n * ld * sizeof (double);
  if (cudaMemsetAsync (P0, 0, blk, s) != cudaSuccess
      || cudaMemsetAsync (P1, 0, blk, s) != cudaSuccess
      || cudaMemsetAsync (R, 0, blk, s) != cudaSuccess
      || cudaMemsetAsync (X, 0, blk, s) != cudaSuccess
      || cudaMemsetAsync (sv->ws.ival.p, 0, sv->ws.ival.n * sizeof (int), s) != cudaSuccess
      || cudaStreamSynchronize (s) != cudaSuccess) {
    srv_fail (sv, set_error (LGH_ERR_GPU, "server: workspace clear"));
    return;
  }
  std::vector<int> act (sv->cap);
  /* one PCG tick over the slot block for a given pair of direction
   * buffers; after two eager ticks (which set up the V-cycle buffers and
   * the launch-shape caches) each parity is captured into a CUDA graph
   * once and replayed, so a tick costs one graph launch on the host.  A
   * mixed-precision object's V-cycle runs in FP32 on rounded copies of the
   * residuals (the FP64 CG scalars and iterates are unchanged). */
  auto tick = [&] (double *Po, double *Pn) -> int {
    if (p->mg && sv->pc32) {
      LGH_TRY ((cvt_flat<double, float> (n * ld, R, R32, s)));
      LGH_TRY (mg_vcycle<float> (p->mg, R32, Z32, ld, sv->cap, s, nullptr, &sv->mgw));
      LGH_TRY ((cvt_flat<float, double> (n * ld, Z32, Zb, s)));
    } else if (p->mg) {
      LGH_TRY (mg_vcycle<double> (p->mg, R, Zb, ld, sv->cap, s, nullptr, &sv->mgw));
    } else {
      LGH_TRY (launch_rowscale<double> (n, ld, p->Z->csr.dinv, R, ld, Zb, ld, s));
    }
    LGH_TRY (server_tick_dots<double> (p->Z->csr, R, Zb, ld, sv->cap, sv->fresh_d.p,
                                       p->zcfg.rtol, sv->ws, s));
    LGH_TRY (server_tick_pq<double> (p->Z->csr, Zb, Po, Pn, Q, ld, sv->ws, s));
    return server_tick_upd<double> (n, ld, X, R, Pn, Q, sv->ws, s);
  };
  cudaGraphExec_t gexec[2] = { nullptr, nullptr };
  bool graphs_off = false;
  int parity = 0;   /* 0: the old direction is in P0 */
  int hold = 0;     /* ticks that converged columns have waited */
  const int batch = std::max (1, sv->cap / 8);
  auto release_graphs = [&] () {
    for (auto &ge : gexec)
      if (ge) { cudaGraphExecDestroy (ge); ge = nullptr; }
  };
  double ta = 0., tt = 0., th = 0.;   /* phase seconds, published per tick */
  double occ = 0.;                    /* occupied slots summed over ticks */
  while (!sv->stop.load () && !sv->failed.load ()) {
    /* 1. admission into free slots */
    double w0 = wall ();
    std::vector<Adm> adm;
    srv_admit (sv, adm);
    for (const Adm &a : adm) {
      rc = (a.r->kind == 2) ? srv_logdet (sv, a.r) : srv_start (sv, a, Pold);
      if (rc) break;
    }
    if (!adm.empty ()) ta += wall () - w0;
    if (rc) { release_graphs (); srv_fail (sv, rc); return; }
    bool any = false;
    for (auto &sl : sv->slots) any |= sl.req != nullptr;
    if (!any) {
      std::unique_lock<std::mutex> lk (sv->mu);
      sv->cv.wait_for (lk, std::chrono::milliseconds (2), [&] {
        return sv->stop.load () || sv->failed.load ()
               || (!sv->pending.empty () && sv->pending.front ()->staged);
      });
      continue;
    }
    /* 2. one PCG tick over the whole slot block: preconditioner, dots
     *    (fresh columns start there), direction + Z product, update */
    w0 = wall ();
    memcpy (sv->fresh_pin, sv->fresh_h.data (), sv->cap * sizeof (int));
    if (cudaMemcpyAsync (sv->fresh_d.p, sv->fresh_pin, sv->cap * sizeof (int),
                         cudaMemcpyHostToDevice, s) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "server: fresh flags");
    if (!rc && !graphs_off && sv->ticks >= 2 && gexec[parity] == nullptr) {
      cudaGraph_t gr = nullptr;
      if (cudaStreamBeginCapture (s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int crc = tick (Pold, Pnew);
        const cudaError_t ce = cudaStreamEndCapture (s, &gr);
        if (crc != 0 || ce != cudaSuccess || gr == nullptr
            || cudaGraphInstantiate (&gexec[parity], gr, 0) != cudaSuccess) {
          gexec[parity] = nullptr;
          graphs_off = true;     /* keep ticking eagerly */
        }
        if (gr) cudaGraphDestroy (gr);
      } else {
        graphs_off = true;
      }
      cudaGetLastError ();
      clear_error ();
    }
    if (!rc) {
      if (gexec[parity]) {
        if (cudaGraphLaunch (gexec[parity], s) != cudaSuccess)
          rc = set_error (LGH_ERR_GPU, "server: tick graph launch");
      } else {
        rc = tick (Pold, Pnew);
      }
    }
    std::swap (Pold, Pnew);
    parity ^= 1;
    std::fill (sv->fresh_h.begin (), sv->fresh_h.end (), 0);
    sv->ticks++;
    /* 3. the convergence mask; converged columns are harvested in
     *    batches (a harvest reads all of U and W once, whatever its
     *    width): at cap/8 columns, when every occupied slot has
     *    converged, or after three ticks of waiting.  A converged column
     *    is frozen (its step lengths are zero), so waiting changes no bit
     *    of its result. */
    if (!rc && cudaMemcpyAsync (sv->act_pin, sv->ws.ival.p, sv->cap * sizeof (int),
                                cudaMemcpyDeviceToHost, s) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "server: mask copy");
    if (!rc && cudaStreamSynchronize (s) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "server: tick");
    tt += wall () - w0;
    if (!rc) {
      memcpy (act.data (), sv->act_pin, sv->cap * sizeof (int));
      int occ_n = 0, conv = 0;
      for (int sl = 0; sl < sv->cap; sl++)
        if (sv->slots[sl].req) {
          occ_n++;
          conv += act[sl] == 0;
        }
      occ += occ_n;
      if (conv > 0) hold++;
      if (conv > 0 && (conv >= batch || conv == occ_n || hold >= 3)) {
        w0 = wall ();
        rc = srv_harvest (sv, act, Pold);
        th += wall () - w0;
        hold = 0;
      }
    }
    {
      std::lock_guard<std::mutex> lk (sv->mu);
      sv->t_admit = ta;
      sv->t_tick = tt;
      sv->t_harvest = th;
      sv->occ_sum = occ;
    }
    if (rc) { release_graphs (); srv_fail (sv, rc); return; }
  }
  release_graphs ();
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

static void
srv_release (lgh_server_t *sv)
{
  if (sv->s) {
    cudaStreamSynchronize (sv->s);
    cudaStreamDestroy (sv->s);
  }
  if (sv->sc) {
    cudaStreamSynchronize (sv->sc);
    cudaStreamDestroy (sv->sc);
  }
  for (auto &kv : sv->reqs)
    if (kv.second->ev_out) cudaEventDestroy (kv.second->ev_out);
  for (auto &e : sv->stg_ev)
    if (e) cudaEventDestroy (e);
  if (sv->stg) cudaFreeHost (sv->stg);
  if (sv->fresh_pin) cudaFreeHost (sv->fresh_pin);
  if (sv->act_pin) cudaFreeHost (sv->act_pin);
  delete sv;
}

int
lgh_server_create (lgh_glr_t *glr, const lgh_server_opts_t *opts,
                   lgh_server_t **out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (glr && out, LGH_ERR_ARG_NULL, "lgh_server_create: NULL");
  LGH_CHECK (glr->prior->is_mat, LGH_ERR_SUP,
             "lgh_server_create: needs a Mat-path prior (device Z-solves)");
  LGH_CHECK (!glr->rows, LGH_ERR_SUP,
             "lgh_server_create: a row-sharded object is served by its "
             "per-call operations");
  lgh_server_opts_t o = opts ? *opts : lgh_server_opts_default ();
  LGH_CHECK (o.slots >= 1 && o.slots <= Harvest::MAXS, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_server_create: slots %d", o.slots);
  lgh_server_t *sv = new lgh_server_t ();
  sv->g = glr;
  sv->cap = o.slots;
  sv->ld = round_ld (o.slots);
  sv->reserve = o.hbm_reserve;
  sv->pc32 = glr->exec.precision == LGH_PREC_MIXED && glr->prior->mg != nullptr;
  int rc = 0;
  if (cudaStreamCreateWithFlags (&sv->s, cudaStreamNonBlocking) != cudaSuccess
      || cudaStreamCreateWithFlags (&sv->sc, cudaStreamNonBlocking) != cudaSuccess)
    rc = set_error (LGH_ERR_GPU, "lgh_server_create: streams");
  /* the shift-independent precompute W = Z^{-1} M^{1/2} U */
  if (!rc) rc = ensure_wz (glr);
  const int kp = std::max (glr->kept, 1);
  if (!rc) rc = sv->ws.alloc (glr->n, sv->ld, 0);
  if (!rc && sv->pc32) {
    rc = sv->ws.R32.alloc ((size_t) glr->n * sv->ld * sizeof (float));
    if (!rc) rc = sv->ws.Z32.alloc ((size_t) glr->n * sv->ld * sizeof (float));
    if (!rc && cudaMemsetAsync (sv->ws.Z32.p, 0, (size_t) glr->n * sv->ld * sizeof (float),
                                sv->s) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "lgh_server_create: clear");
  }
  if (!rc) rc = sv->fresh_d.alloc (sv->ld);
  if (!rc) rc = sv->H.alloc ((size_t) glr->n * sv->ld);
  if (!rc) rc = sv->coef.alloc ((size_t) kp * sv->cap);
  /* the harvests' U^T products run at every width up to the slot count */
  if (!rc) rc = sv->gemmwork.alloc (std::max<size_t> (
             gemm_tn_work_max (kp, sv->cap), 64));
  if (!rc) rc = sv->ldc.alloc (1);
  if (!rc) rc = sv->ldo.alloc (1);
  if (!rc) rc = sv->hv_d.alloc (sizeof (Harvest));
  if (!rc && (cudaMallocHost ((void **) &sv->fresh_pin, sv->ld * sizeof (int)) != cudaSuccess
              || cudaMallocHost ((void **) &sv->act_pin, sv->ld * sizeof (int)) != cudaSuccess))
    rc = set_error (LGH_ERR_MEM, "lgh_server_create: pinned buffers");
  /* staging halves of at least one column and 32 MiB */
  sv->stg_half = std::max<size_t> ((size_t) 32 << 20, (size_t) glr->n * 8);
  if (!rc && cudaMallocHost ((void **) &sv->stg, 2 * sv->stg_half) != cudaSuccess)
    rc = set_error (LGH_ERR_MEM, "lgh_server_create: staging buffers");
  for (auto &e : sv->stg_ev)
    if (!rc && (cudaEventCreateWithFlags (&e, cudaEventDisableTiming) != cudaSuccess
                || cudaEventRecord (e, sv->sc) != cudaSuccess))
      rc = set_error (LGH_ERR_GPU, "lgh_server_create: staging events");
  if (!rc) rc = cudaDeviceSynchronize () == cudaSuccess ? 0
                : set_error (LGH_ERR_GPU, "lgh_server_create: set-up");
  if (rc) {
    srv_release (sv);
    return rc;
  }
  sv->hv.reset (new Harvest ());
  sv->slots.assign (sv->cap, Slot ());
  sv->fresh_h.assign (sv->ld, 0);
  sv->t0 = wall ();
  int dev = 0;
  cudaGetDevice (&dev);
  sv->worker = std::thread ([sv, dev] {
    cudaSetDevice (dev);
    srv_loop (sv);
  });
  sv->copier = std::thread ([sv, dev] {
    cudaSetDevice (dev);
    srv_copier (sv);
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
    LGH_CHECK (in && out && m >= 1 && ldin >= sv->g->n && ldout >= sv->g->n,
               LGH_ERR_ARG_SIZ, "lgh_server_submit: need m >= 1 and ld >= n");
  }
  std::unique_ptr<SReq> r (new SReq ());
  r->kind = kind;
  r->c = c;
  r->m = kind == 2 ? 0 : m;
  r->hin = in;
  r->ldin = ldin;
  r->hout = out;
  r->ldout = ldout;
  r->staged = kind == 2;
  r->t_submit = wall ();
  std::lock_guard<std::mutex> lk (sv->mu);
  LGH_CHECK (sv->err == 0, sv->err, "lgh_server_submit: server failed: %s",
             sv->errmsg.c_str ());
  r->id = sv->next_id++;
  *id = r->id;
  sv->pending.push_back (r.get ());
  if (kind != 2) sv->up_q.push_back (r.get ());
  sv->reqs[r->id] = std::move (r);
  sv->cv.notify_all ();
  sv->ccv.notify_all ();
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
  if (r->status < 0) {
    const int code = -r->status;
    sv->reqs.erase (it);
    return set_error (code, "lgh_server_wait: request failed%s%s",
                      sv->errmsg.empty () ? "" : ": ", sv->errmsg.c_str ());
  }
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
  st->t_admit_s = sv->t_admit;
  st->t_tick_s = sv->t_tick;
  st->t_harvest_s = sv->t_harvest;
  st->harvests = sv->harvests;
  st->t_up_s = sv->t_up;
  st->t_down_s = sv->t_down;
  st->occupancy = sv->ticks > 0 ? sv->occ_sum / ((double) sv->ticks * sv->cap) : 0.;
  if (sv->st_n > 0) {
    st->wait_stage_s = sv->st_stage / sv->st_n;
    st->wait_admit_s = sv->st_admit / sv->st_n;
    st->run_s = sv->st_run / sv->st_n;
    st->copy_out_s = sv->st_out / sv->st_n;
  }
  return 0;
}

void
lgh_server_destroy (lgh_server_t *sv)
{
  if (!sv) return;
  sv->stop.store (true);
  {
    std::lock_guard<std::mutex> lk (sv->mu);
    sv->cv.notify_all ();
    sv->ccv.notify_all ();
  }
  if (sv->worker.joinable ()) sv->worker.join ();
  if (sv->copier.joinable ()) sv->copier.join ();
  srv_release (sv);
}

} /* extern "C" */
