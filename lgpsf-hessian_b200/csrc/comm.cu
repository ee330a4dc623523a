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
 *
 * lgh_rows_local_create gives the same for the build over row slabs: an
 * all-reduce (host-staged, summed in rank order, so identical on every
 * rank) and the halo all-to-all (device to device copies of each peer's
 * chunk).
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
  std::vector<const size_t *> posted_bytes;     /* row slabs: per-peer sizes */
  std::vector<std::vector<double>> stage;       /* row slabs: all-reduce     */
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

/* row slabs: every rank stages its buffer on the host, all ranks sum the
 * stages in rank order (the same additions on every rank, so the same
 * result), then wait before a stage may be overwritten */
int
local_allreduce (double *buf, size_t count, void *ctx)
{
  RankCtx *rc = (RankCtx *) ctx;
  Shared *sh = rc->sh;
  std::vector<double> &mine = sh->stage[rc->rank];
  mine.resize (count);
  if (cudaMemcpy (mine.data (), buf, count * sizeof (double),
                  cudaMemcpyDeviceToHost) != cudaSuccess)
    return 2;
  if (!meet (sh)) return 1;
  std::vector<double> sum (count, 0.);
  int rcode = 0;
  for (int r = 0; r < sh->size; r++) {
    if (sh->stage[r].size () != count) rcode = 3;
    else
      for (size_t i = 0; i < count; i++) sum[i] += sh->stage[r][i];
  }
  if (!rcode && cudaMemcpy (buf, sum.data (), count * sizeof (double),
                            cudaMemcpyHostToDevice) != cudaSuccess)
    rcode = 2;
  if (!meet (sh)) return 1;
  return rcode;
}

/* row slabs: each rank copies its chunk of every peer's send buffer (the
 * peer's per-peer sizes give the offset) device to device */
int
local_alltoallv (const void *send, const size_t *send_bytes, void *recv,
                 const size_t *recv_bytes, void *ctx)
{
  RankCtx *rc = (RankCtx *) ctx;
  Shared *sh = rc->sh;
  const int me = rc->rank;
  {
    std::lock_guard<std::mutex> lk (sh->mu);
    sh->posted[me] = send;
    sh->posted_bytes[me] = send_bytes;
  }
  if (!meet (sh)) return 1;
  int rcode = 0;
  size_t roff = 0;
  for (int p = 0; p < sh->size && !rcode; p++) {
    const size_t *pb = sh->posted_bytes[p];
    size_t soff = 0;
    for (int q = 0; q < me; q++) soff += pb[q];
    if (pb[me] != recv_bytes[p]) rcode = 3;
    else if (recv_bytes[p] > 0
             && cudaMemcpy ((char *) recv + roff,
                            (const char *) sh->posted[p] + soff, recv_bytes[p],
                            cudaMemcpyDeviceToDevice) != cudaSuccess)
      rcode = 2;
    roff += recv_bytes[p];
  }
  if (!meet (sh)) return 1;
  return rcode;
}

Shared *
new_shared (int size)
{
  Shared *sh = new Shared ();
  sh->size = size;
  sh->posted.assign (size, nullptr);
  sh->posted_bytes.assign (size, nullptr);
  sh->stage.assign (size, {});
  return sh;
}

} /* namespace */

extern "C" {

int
lgh_comm_local_create (int size, lgh_comm_t *comms)
{
  LGH_CHECK (comms && size >= 1 && size <= 64, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_comm_local_create: size %d (1 .. 64)", size);
  Shared *sh = new_shared (size);
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

int
lgh_rows_local_create (int size, lgh_rows_comm_t *comms)
{
  LGH_CHECK (comms && size >= 1 && size <= 64, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_rows_local_create: size %d (1 .. 64)", size);
  Shared *sh = new_shared (size);
  for (int r = 0; r < size; r++) {
    comms[r].rank = r;
    comms[r].size = size;
    comms[r].allreduce = &local_allreduce;
    comms[r].alltoallv = &local_alltoallv;
    comms[r].ctx = new RankCtx{ sh, r };
  }
  return 0;
}

void
lgh_rows_local_destroy (lgh_rows_comm_t *comms)
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
