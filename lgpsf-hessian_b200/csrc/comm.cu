/* comm.cu -- the in-process communicator of the column-sharded build.
 *
 * lgh_comm_local_create gives `size` communicators for ranks that run as
 * threads of one process on one device.  Their all-gather meets on a host
 * barrier: every rank posts its send buffer, waits for the others, copies
 * all posted buffers device to device into its own receive buffer, and
 * waits again before any rank may reuse its send buffer.  Kernels never
 * wait for another rank (the ranks' launches serialise on the device); a
 * rank that does not arrive within the time limit makes the others' call
 * return an error instead of waiting for good.  Multi-process runs pass a
 * communicator of their own (for example over NCCL).
 */

#include <chrono>
#include <condition_variable>
#include <mutex>
#include <vector>

#include "lgh_internal.h"

namespace
{

struct Shared
{
  int size = 0;
  std::mutex mu;
  std::condition_variable cv;
  int arrived = 0;
  long generation = 0;
  std::vector<const void *> posted;
  bool broken = false;
};

struct RankCtx
{
  Shared *sh;
  int rank;
};

/* a reusable barrier with a time limit; false when it ran out */
bool
meet (Shared *sh)
{
  std::unique_lock<std::mutex> lk (sh->mu);
  if (sh->broken) return false;
  const long gen = sh->generation;
  if (++sh->arrived == sh->size) {
    sh->arrived = 0;
    sh->generation++;
    sh->cv.notify_all ();
    return true;
  }
  const bool ok = sh->cv.wait_for (lk, std::chrono::seconds (120),
                                   [&] { return sh->generation != gen || sh->broken; });
  if (!ok || sh->broken) {
    sh->broken = true;
    sh->cv.notify_all ();
    return false;
  }
  return true;
}

int
local_allgather (const void *send, void *recv, size_t len, void *ctx)
{
  RankCtx *rc = (RankCtx *) ctx;
  Shared *sh = rc->sh;
  {
    std::lock_guard<std::mutex> lk (sh->mu);
    sh->posted[rc->rank] = send;
  }
  if (!meet (sh)) return 1;
  for (int r = 0; r < sh->size; r++)
    if (cudaMemcpy ((char *) recv + (size_t) r * len, sh->posted[r], len,
                    cudaMemcpyDeviceToDevice) != cudaSuccess)
      return 2;
  return meet (sh) ? 0 : 1;
}

} /* namespace */

extern "C" {

int
lgh_comm_local_create (int size, lgh_comm_t *comms)
{
  LGH_CHECK (comms && size >= 1 && size <= 64, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_comm_local_create: size %d (1 .. 64)", size);
  Shared *sh = new Shared ();
  sh->size = size;
  sh->posted.assign (size, nullptr);
  for (int r = 0; r < size; r++) {
    RankCtx *rc = new RankCtx{ sh, r };
    comms[r].rank = r;
    comms[r].size = size;
    comms[r].send = nullptr;
    comms[r].recv = nullptr;
    comms[r].bytes = 0;
    comms[r].allgather = &local_allgather;
    comms[r].ctx = rc;
  }
  return 0;
}

void
lgh_comm_local_destroy (lgh_comm_t *comms)
{
  if (!comms || !comms[0].ctx) return;
  const int size = comms[0].size;
  Shared *sh = ((RankCtx *) comms[0].ctx)->sh;
  for (int r = 0; r < size; r++) {
    delete (RankCtx *) comms[r].ctx;
    comms[r].ctx = nullptr;
  }
  delete sh;
}

} /* extern "C" */
