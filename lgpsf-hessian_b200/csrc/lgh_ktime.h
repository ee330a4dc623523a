/* lgh_ktime.h -- per-kernel CUDA-event timing (see ktime.cu). */

#ifndef LGH_KTIME_H
#define LGH_KTIME_H

#include <cuda_runtime.h>

#include <vector>

namespace lgh
{

enum KId { K_PCG_PQ = 0, K_PCG_UPD, K_CHEB, K_SPMM, K_PCG_INIT, K_NKERN };

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

} /* namespace lgh */

#endif /* LGH_KTIME_H */
