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
 * all-reduce (every rank sums all ranks' device buffers in rank order, so
 * the result is identical on every rank) and the halo all-to-all (device
 * to device copies of each peer's chunk).
 */

#include <algorithm>
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
  double *sum = nullptr;        /* row slabs: this rank's all-reduce scratch */
  size_t sum_n = 0;
};

/* y[i] += x[i] */
__global__ void
k_local_add (size_t n, const double *__restrict__ x, double *__restrict__ y)
{
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t) gridDim.x * blockDim.x)
    y[i] += x[i];
}

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

/* row slabs: every rank posts its device buffer; each rank sums all
 * posted buffers in rank order into its scratch on the device (the same
 * additions on every rank, so the same result), waits until every rank
 * has read every buffer, and only then overwrites its own */
int
local_allreduce (double *buf, size_t count, void *ctx)
{
  RankCtx *rc = (RankCtx *) ctx;
  Shared *sh = rc->sh;
  int rcode = 0;
  if (rc->sum_n < count) {
    cudaFree (rc->sum);
    rc->sum = nullptr;
    rc->sum_n = 0;
    if (cudaMalloc ((void **) &rc->sum, count * sizeof (double)) == cudaSuccess)
      rc->sum_n = count;
    else
      rcode = 2;
  }
  {
    std::lock_guard<std::mutex> lk (sh->mu);
    sh->posted[rc->rank] = buf;
    sh->stage[rc->rank].assign (1, (double) count);
  }
  if (!meet (sh)) return 1;
  for (int r = 0; r < sh->size && !rcode; r++)
    if (sh->stage[r].size () != 1 || sh->stage[r][0] != (double) count) rcode = 3;
  if (!rcode) {
    const int grid = (int) std::min<size_t> ((count + 255) / 256, 4096);
    if (cudaMemcpy (rc->sum, sh->posted[0], count * sizeof (double),
                    cudaMemcpyDeviceToDevice) != cudaSuccess)
      rcode = 2;
    for (int r = 1; r < sh->size && !rcode; r++) {
      k_local_add<<<grid > 0 ? grid : 1, 256>>> (count,
                                                 (const double *) sh->posted[r],
                                                 rc->sum);
      if (cudaGetLastError () != cudaSuccess) rcode = 2;
    }
    if (!rcode && cudaDeviceSynchronize () != cudaSuccess) rcode = 2;
  }
  if (!meet (sh)) return 1;
  if (!rcode && cudaMemcpy (buf, rc->sum, count * sizeof (double),
                            cudaMemcpyDeviceToDevice) != cudaSuccess)
    rcode = 2;
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
    RankCtx *rc = (RankCtx *) comms[r].ctx;
    if (rc) cudaFree (rc->sum);
    delete rc;
    comms[r].ctx = nullptr;
  }
  delete sh;
}

} /* extern "C" */
