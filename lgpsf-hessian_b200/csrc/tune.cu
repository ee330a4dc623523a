/* tune.cu -- the library's autotuner.
 *
 * A tunable operation offers a few launch variants (tile shapes) that
 * compute the same result.  The first call of a shape key runs each
 * variant once, timed with CUDA events on the library's stream, and keeps
 * the fastest; later calls of that key look the choice up.  The choices
 * live in a process-wide table and, when LGH_TUNE_CACHE names a file, in
 * that file too (read on first use, one line appended per new key:
 * "op n kept m nshift variant ms"), so a serving process that restarts
 * does not tune again.  A file entry that names a variant out of range is
 * ignored.
 */

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "lgh_batch.h"
#include "lgh_internal.h"

namespace lgh
{

namespace
{

typedef std::tuple<std::string, int64_t, int, int, int> Key;

std::mutex g_mu;
std::map<Key, int> g_table;
bool g_loaded = false;

void
load_cache ()
{
  if (g_loaded) return;
  g_loaded = true;
  const char *path = getenv ("LGH_TUNE_CACHE");
  if (!path || !*path) return;
  FILE *f = fopen (path, "r");
  if (!f) return;
  char op[64];
  long long n;
  int kept, m, ns, v;
  double ms;
  while (fscanf (f, "%63s %lld %d %d %d %d %lf", op, &n, &kept, &m, &ns, &v,
                 &ms) == 7)
    g_table[Key (op, (int64_t) n, kept, m, ns)] = v;
  fclose (f);
}

void
save_entry (const Key &k, int v, double ms)
{
  const char *path = getenv ("LGH_TUNE_CACHE");
  if (!path || !*path) return;
  FILE *f = fopen (path, "a");
  if (!f) return;
  fprintf (f, "%s %lld %d %d %d %d %.6f\n", std::get<0> (k).c_str (),
           (long long) std::get<1> (k), std::get<2> (k), std::get<3> (k),
           std::get<4> (k), v, ms);
  fclose (f);
}

} /* namespace */

int
tune_pick (const char *op, int64_t n, int kept, int m, int nshift,
           int nvariants, tune_trial_fn trial, void *ctx, int *variant,
           int *measured)
{
  const Key key (op, n, kept, m, nshift);
  *measured = 0;
  {
    std::lock_guard<std::mutex> lk (g_mu);
    load_cache ();
    auto it = g_table.find (key);
    if (it != g_table.end () && it->second >= 0 && it->second < nvariants) {
      *variant = it->second;
      return 0;
    }
  }
  cudaStream_t s = stream ();
  cudaEvent_t e0, e1;
  LGH_CUDA (cudaEventCreate (&e0));
  LGH_CUDA (cudaEventCreate (&e1));
  int best = 0;
  float best_ms = 0.f;
  int rc = 0;
  /* each variant twice, the faster run kept: a variant's first launch also
   * loads its module, which is no part of its speed */
  for (int v = 0; v < nvariants && !rc; v++) {
    for (int rep = 0; rep < 2 && !rc; rep++) {
      if (cudaEventRecord (e0, s) != cudaSuccess) { rc = set_error (LGH_ERR_GPU, "tune: event"); break; }
      rc = trial (v, ctx);
      if (rc) break;
      if (cudaEventRecord (e1, s) != cudaSuccess
          || cudaEventSynchronize (e1) != cudaSuccess) {
        rc = set_error (LGH_ERR_GPU, "tune: event");
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime (&ms, e0, e1);
      if ((v == 0 && rep == 0) || ms < best_ms) { best = v; best_ms = ms; }
    }
  }
  cudaEventDestroy (e0);
  cudaEventDestroy (e1);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk (g_mu);
    g_table[key] = best;
    save_entry (key, best, best_ms);
  }
  *variant = best;
  *measured = 1;
  return 0;
}

int
tune_table_size ()
{
  std::lock_guard<std::mutex> lk (g_mu);
  return (int) g_table.size ();
}

} /* namespace lgh */
