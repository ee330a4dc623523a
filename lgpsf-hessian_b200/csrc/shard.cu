/* shard.cu -- row-sharded operators for more than one GPU.
 *
 * The reference distributes every vector and sparse operator over its MPI
 * ranks in contiguous row slabs (PETSc's MPIAIJ / MPIDENSE layout; the
 * Woodbury recipe runs on those slabs, docs/glr-woodbury-formulas.tex:
 * 76-98): B X and the Z-solves need the rows of X owned by other ranks that
 * the local nonzeros reference (the ghost rows, PETSc's VecScatter of
 * MatMult), and every Gram / Q^T Y / U^T X is a local product plus one
 * all-reduce.  A shard plan is one rank's view of a symmetric CSR operator:
 *
 *   owned rows [row0, row1) of N (the even split r N / P);
 *   ghost rows: the remote global rows its nonzeros reference, ascending,
 *     with the number owned by each rank (contiguous runs, since ranks own
 *     contiguous ranges);
 *   local column indices: owned column c -> c - row0, ghost g -> nloc +
 *     its position in the ghost list, so the local operator multiplies an
 *     extended row-major block [owned rows; ghost rows];
 *   sends: for each peer, the owned rows the peer listed as its ghosts
 *     (registered after the caller's all-to-all of the ghost lists).
 *
 * The exchange itself is the caller's collective (NCCL or gloo send /
 * receive of contiguous buffers); lgh_shard_pack gathers a peer's send rows
 * of a block into a contiguous buffer and lgh_shard_unpack writes a
 * received buffer into the ghost rows of the extended block (device
 * kernels).  The plan is host code and touches no device memory until the
 * first pack.
 */

#include <string.h>

#include <algorithm>
#include <vector>

#include "lgh_device.cuh"
#include "lgh_internal.h"

struct lgh_shard
{
  int64_t N = 0, row0 = 0, row1 = 0;
  int nranks = 1, rank = 0;
  std::vector<int64_t> starts;          /* rank r owns [starts[r], starts[r+1]) */
  std::vector<int64_t> ghosts;          /* ascending global rows            */
  std::vector<int64_t> ghost_count;     /* per owner rank                   */
  std::vector<int64_t> ghost_first;     /* offset of each owner's run       */
  std::vector<int32_t> lcol;            /* local column indices             */
  std::vector<std::vector<int64_t>> sends; /* per peer, local owned rows    */
  std::vector<lgh::DBuf<int64_t>> dsends;  /* device copies (lazy)          */
};

namespace lgh
{

static void
shard_range (int64_t N, int P, int r, int64_t *a, int64_t *b)
{
  *a = (int64_t) ((__int128) N * r / P);
  *b = (int64_t) ((__int128) N * (r + 1) / P);
}

static int
shard_owner (const lgh_shard_t *sh, int64_t g)
{
  /* the last r with starts[r] <= g (empty ranks own nothing) */
  const auto it = std::upper_bound (sh->starts.begin (), sh->starts.end (), g);
  return (int) (it - sh->starts.begin ()) - 1;
}

/* rows of X listed in idx -> contiguous buf (count x w, row stride w) */
__global__ void
k_shard_pack (int64_t count, int w, const int64_t *idx, const double *X,
              int64_t ldx, double *buf)
{
  const int64_t total = count * w;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t r = e / w;
    const int c = (int) (e - r * w);
    buf[e] = X[idx[r] * ldx + c];
  }
}

/* contiguous buf -> rows first .. first+count-1 of the extended block */
__global__ void
k_shard_unpack (int64_t count, int w, const double *buf, double *X,
                int64_t ld, int64_t first)
{
  const int64_t total = count * w;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t r = e / w;
    const int c = (int) (e - r * w);
    X[(first + r) * ld + c] = buf[e];
  }
}

static int
shard_grid (int64_t total)
{
  int64_t g = (total + 255) / 256;
  const int64_t cap = (int64_t) num_sms () * 8;
  if (g > cap) g = cap;
  return (int) (g > 0 ? g : 1);
}

/* the plan for an explicit contiguous partition: rank r owns rows
 * [starts[r], starts[r + 1]), starts[0] = 0, starts[nranks] = N,
 * non-decreasing */
int
shard_create_ranges (int64_t N, int nranks, int rank, const int64_t *starts,
                     const int64_t *rowptr, const int32_t *colidx,
                     lgh_shard_t **out)
{
  LGH_CHECK (rowptr && out && starts, LGH_ERR_ARG_NULL,
             "lgh_shard_create: NULL argument");
  LGH_CHECK (N >= 1 && nranks >= 1 && rank >= 0 && rank < nranks,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_shard_create: N %lld, rank %d of %d",
             (long long) N, rank, nranks);
  LGH_CHECK (starts[0] == 0 && starts[nranks] == N, LGH_ERR_ARG_WRONG,
             "lgh_shard_create: the ranks' rows must cover [0, %lld)",
             (long long) N);
  for (int r = 0; r < nranks; r++)
    LGH_CHECK (starts[r] <= starts[r + 1], LGH_ERR_ARG_WRONG,
               "lgh_shard_create: rank %d's rows are not contiguous after "
               "rank %d's", r + 1, r);
  lgh_shard_t *sh = new lgh_shard_t ();
  sh->N = N;
  sh->nranks = nranks;
  sh->rank = rank;
  sh->starts.assign (starts, starts + nranks + 1);
  sh->row0 = starts[rank];
  sh->row1 = starts[rank + 1];
  const int64_t nloc = sh->row1 - sh->row0;
  const int64_t nnz = rowptr[nloc] - rowptr[0];
  if (nnz > 0 && colidx == nullptr) {
    delete sh;
    return set_error (LGH_ERR_ARG_NULL, "lgh_shard_create: NULL colidx");
  }
  /* ghosts: remote columns, deduplicated and sorted */
  std::vector<int64_t> g;
  for (int64_t k = 0; k < nnz; k++) {
    const int64_t c = colidx[k];
    if (c < 0 || c >= N) {
      delete sh;
      return set_error (LGH_ERR_ARG_OUTOFRANGE,
                        "lgh_shard_create: column %lld outside [0, %lld)",
                        (long long) c, (long long) N);
    }
    if (c < sh->row0 || c >= sh->row1) g.push_back (c);
  }
  std::sort (g.begin (), g.end ());
  g.erase (std::unique (g.begin (), g.end ()), g.end ());
  sh->ghosts = g;
  sh->ghost_count.assign (nranks, 0);
  sh->ghost_first.assign (nranks, 0);
  for (int64_t x : g) sh->ghost_count[shard_owner (sh, x)]++;
  for (int r = 1; r < nranks; r++)
    sh->ghost_first[r] = sh->ghost_first[r - 1] + sh->ghost_count[r - 1];
  /* local column numbering over [owned; ghosts] */
  sh->lcol.resize (nnz);
  for (int64_t k = 0; k < nnz; k++) {
    const int64_t c = colidx[k];
    if (c >= sh->row0 && c < sh->row1) {
      sh->lcol[k] = (int32_t) (c - sh->row0);
    } else {
      const int64_t pos = std::lower_bound (g.begin (), g.end (), c) - g.begin ();
      sh->lcol[k] = (int32_t) (nloc + pos);
    }
  }
  sh->sends.assign (nranks, {});
  sh->dsends.resize (nranks);
  *out = sh;
  return 0;
}

} /* namespace lgh */

using namespace lgh;

extern "C" {

void
lgh_shard_range (int64_t N, int nranks, int rank, int64_t *row0, int64_t *row1)
{
  if (nranks < 1 || rank < 0 || rank >= nranks) {
    *row0 = *row1 = 0;
    return;
  }
  shard_range (N, nranks, rank, row0, row1);
}

int
lgh_shard_create (int64_t N, int nranks, int rank, const int64_t *rowptr,
                  const int32_t *colidx, lgh_shard_t **out)
{
  LGH_CHECK (N >= 1 && nranks >= 1 && rank >= 0 && rank < nranks,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_shard_create: N %lld, rank %d of %d",
             (long long) N, rank, nranks);
  std::vector<int64_t> st (nranks + 1);
  for (int r = 0; r < nranks; r++) {
    int64_t a, b;
    shard_range (N, nranks, r, &a, &b);
    st[r] = a;
    st[r + 1] = b;
  }
  return lgh::shard_create_ranges (N, nranks, rank, st.data (), rowptr, colidx,
                                   out);
}

int
lgh_shard_info (const lgh_shard_t *sh, int64_t *row0, int64_t *row1,
                int64_t *nghost)
{
  LGH_CHECK (sh, LGH_ERR_ARG_NULL, "lgh_shard_info: NULL");
  if (row0) *row0 = sh->row0;
  if (row1) *row1 = sh->row1;
  if (nghost) *nghost = (int64_t) sh->ghosts.size ();
  return 0;
}

int
lgh_shard_ghosts (const lgh_shard_t *sh, const int64_t **rows,
                  const int64_t **counts)
{
  LGH_CHECK (sh && rows && counts, LGH_ERR_ARG_NULL, "lgh_shard_ghosts: NULL");
  *rows = sh->ghosts.data ();
  *counts = sh->ghost_count.data ();
  return 0;
}

int
lgh_shard_local_colidx (const lgh_shard_t *sh, const int32_t **colidx)
{
  LGH_CHECK (sh && colidx, LGH_ERR_ARG_NULL, "lgh_shard_local_colidx: NULL");
  *colidx = sh->lcol.data ();
  return 0;
}

int
lgh_shard_set_sends (lgh_shard_t *sh, int peer, int64_t count,
                     const int64_t *rows)
{
  LGH_CHECK (sh && (rows || count == 0), LGH_ERR_ARG_NULL,
             "lgh_shard_set_sends: NULL");
  LGH_CHECK (peer >= 0 && peer < sh->nranks && peer != sh->rank && count >= 0,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_shard_set_sends: peer %d", peer);
  std::vector<int64_t> loc (count);
  for (int64_t k = 0; k < count; k++) {
    LGH_CHECK (rows[k] >= sh->row0 && rows[k] < sh->row1, LGH_ERR_ARG_WRONG,
               "lgh_shard_set_sends: row %lld is not owned by rank %d",
               (long long) rows[k], sh->rank);
    loc[k] = rows[k] - sh->row0;
  }
  sh->sends[peer] = loc;
  sh->dsends[peer].release ();
  return 0;
}

int
lgh_shard_sends (const lgh_shard_t *sh, int peer, int64_t *count,
                 const int64_t **local_rows)
{
  LGH_CHECK (sh && count && local_rows, LGH_ERR_ARG_NULL,
             "lgh_shard_sends: NULL");
  LGH_CHECK (peer >= 0 && peer < sh->nranks, LGH_ERR_ARG_OUTOFRANGE,
             "lgh_shard_sends: peer %d", peer);
  *count = (int64_t) sh->sends[peer].size ();
  *local_rows = sh->sends[peer].data ();
  return 0;
}

int
lgh_shard_pack (lgh_shard_t *sh, int peer, int w, const double *X, int64_t ldx,
                double *buf)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (sh && X && buf, LGH_ERR_ARG_NULL, "lgh_shard_pack: NULL");
  LGH_CHECK (peer >= 0 && peer < sh->nranks && w >= 1 && ldx >= w,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_shard_pack: peer %d, w %d", peer, w);
  const std::vector<int64_t> &v = sh->sends[peer];
  if (v.empty ()) return 0;
  DBuf<int64_t> &d = sh->dsends[peer];
  cudaStream_t s = stream ();
  if (d.p == nullptr) {
    LGH_TRY (d.alloc (v.size ()));
    LGH_CUDA (cudaMemcpyAsync (d.p, v.data (), v.size () * sizeof (int64_t),
                               cudaMemcpyHostToDevice, s));
  }
  const int64_t cnt = (int64_t) v.size ();
  k_shard_pack<<<shard_grid (cnt * w), 256, 0, s>>> (cnt, w, d.p, X, ldx, buf);
  LGH_LAUNCH_CHECK ();
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

int
lgh_shard_unpack (const lgh_shard_t *sh, int peer, int w, const double *buf,
                  double *Xext, int64_t ld)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (sh && buf && Xext, LGH_ERR_ARG_NULL, "lgh_shard_unpack: NULL");
  LGH_CHECK (peer >= 0 && peer < sh->nranks && w >= 1 && ld >= w,
             LGH_ERR_ARG_OUTOFRANGE, "lgh_shard_unpack: peer %d, w %d", peer, w);
  const int64_t cnt = sh->ghost_count[peer];
  if (cnt == 0) return 0;
  const int64_t first = (sh->row1 - sh->row0) + sh->ghost_first[peer];
  cudaStream_t s = stream ();
  k_shard_unpack<<<shard_grid (cnt * w), 256, 0, s>>> (cnt, w, buf, Xext, ld,
                                                       first);
  LGH_LAUNCH_CHECK ();
  LGH_CUDA (cudaStreamSynchronize (s));
  return 0;
}

void
lgh_shard_destroy (lgh_shard_t *sh)
{
  delete sh;
}

} /* extern "C" */
