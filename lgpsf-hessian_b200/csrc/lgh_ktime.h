/* lgh_ktime.h -- per-kernel CUDA-event timing (see ktime.cu). */

#ifndef LGH_KTIME_H
#define LGH_KTIME_H

#include <cuda_runtime.h>

#include <vector>

namespace lgh
{

enum KId
{
  K_PCG_PQ = 0, K_PCG_UPD, K_CHEB, K_SPMM, K_PCG_INIT,
  K_PCGX_PQ, K_PCGX_UPD, K_PCGX_DOTS, K_CHEBX,
  K_MG_SMOOTH, K_MG_RESID, K_MG_RESTRICT, K_MG_PROLONG, K_MG_COARSE,
  K_MG_TAIL, K_PCGX_PFORM, K_MG_FIRST, K_MG_POST, K_MG_POSTP,
  K_NKERN
};

/* pending event pairs of one stream: ids[i] names the interval between
 * event i and event i + 1 (-1 = not a kernel) */
struct KTrace;

int ktime_on ();
void ktime_add (int id, double ms, double bytes);

/* a growable pool of events recorded in order on one stream */
struct EventRing
{
  std::vector<cudaEvent_t> ev;
  int used = 0;
  int record (cudaStream_t s);
  int drain (const std::vector<int> &ids, const std::vector<double> &bytes);
  ~EventRing ();
};

struct KTrace
{
  EventRing ring;
  std::vector<int> ids;
  std::vector<double> bytes;
  /* start an interval (kernel id and its algorithmic bytes) */
  int begin (int id, double b, cudaStream_t s)
  {
    int rc = ring.record (s);
    ids.push_back (id);
    bytes.push_back (b);
    return rc;
  }
  /* close the current interval */
  int end (cudaStream_t s)
  {
    int rc = ring.record (s);
    ids.push_back (-1);
    bytes.push_back (0.);
    return rc;
  }
  /* after a synchronisation of the stream */
  int drain ()
  {
    int rc = ring.drain (ids, bytes);
    ids.clear ();
    bytes.clear ();
    return rc;
  }
};

} /* namespace lgh */

#endif /* LGH_KTIME_H */
