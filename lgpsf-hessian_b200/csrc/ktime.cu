/* ktime.cu -- optional CUDA-event timing of the hot kernels.
 *
 * When switched on (lgh_kernel_timing(1)), the Z-solve loop and the B
 * product record an event pair around every launch of the kernels below,
 * on the stream they run on, and accumulate the elapsed device time at the
 * solver's existing synchronisation points.  Used by the benchmark to
 * report each kernel's average launch duration for the roofline.
 */

#include <mutex>
#include <vector>

#include "lgh_internal.h"
#include "lgh_ktime.h"

namespace lgh
{

static int g_on = 0;
static std::mutex g_mu;
static double g_ms[K_NKERN];
static long g_n[K_NKERN];
static double g_bytes[K_NKERN];

static const char *g_names[K_NKERN] = {
  "k_pcg_pq", "k_pcg_upd", "k_cheb", "k_spmm", "k_pcg_init",
  "k_pcgx_pq", "k_pcgx_upd", "k_pcgx_dots", "k_chebx",
  "k_cheb@vcycle", "k_spmm<resid>@vcycle", "k_spmm@restrict",
  "k_spmm<acc>@prolong", "k_dense_apply@coarse", "k_cheb_tail@vcycle",
  "k_pcgx_pform", "k_spmm<first>@vcycle",
  "k_spmm<post>@vcycle",
  "k_post_prolong@vcycle"
};

int
ktime_on ()
{
  return g_on;
}

void
ktime_add (int id, double ms, double bytes)
{
  std::lock_guard<std::mutex> lk (g_mu);
  g_ms[id] += ms;
  g_n[id] += 1;
  g_bytes[id] += bytes;
}

int
EventRing::record (cudaStream_t s)
{
  if (used >= (int) ev.size ()) {
    cudaEvent_t e;
    LGH_CUDA (cudaEventCreate (&e));
    ev.push_back (e);
  }
  LGH_CUDA (cudaEventRecord (ev[used], s));
  used++;
  return 0;
}

/* consecutive pairs (ev[i], ev[i+1]) -> kernel ids[i] ; needs a prior sync */
int
EventRing::drain (const std::vector<int> &ids, const std::vector<double> &bytes)
{
  for (size_t i = 0; i + 1 < (size_t) used && i < ids.size (); i++) {
    if (ids[i] < 0) continue;
    float ms = 0.f;
    LGH_CUDA (cudaEventElapsedTime (&ms, ev[i], ev[i + 1]));
    ktime_add (ids[i], ms, bytes[i]);
  }
  used = 0;
  return 0;
}

EventRing::~EventRing ()
{
  for (auto e : ev) cudaEventDestroy (e);
}

} /* namespace lgh */

extern "C" {

/* Switch per-kernel event timing on (1) or off (0); switching resets the
 * accumulated figures. */
int
lgh_kernel_timing (int on)
{
  std::lock_guard<std::mutex> lk (lgh::g_mu);
  lgh::g_on = on;
  for (int i = 0; i < lgh::K_NKERN; i++) {
    lgh::g_ms[i] = 0.;
    lgh::g_n[i] = 0;
    lgh::g_bytes[i] = 0.;
  }
  return 0;
}

/* Accumulated device milliseconds, launches and algorithmic bytes of
 * kernel id (0 k_pcg_pq, 1 k_pcg_upd, 2 k_cheb, 3 k_spmm (B), 4
 * k_pcg_init); returns the kernel's name, or NULL past the last id. */
const char *
lgh_kernel_timing_get (int id, double *ms, long *launches, double *bytes)
{
  if (id < 0 || id >= lgh::K_NKERN) return nullptr;
  std::lock_guard<std::mutex> lk (lgh::g_mu);
  if (ms) *ms = lgh::g_ms[id];
  if (launches) *launches = lgh::g_n[id];
  if (bytes) *bytes = lgh::g_bytes[id];
  return lgh::g_names[id];
}

} /* extern "C" */
