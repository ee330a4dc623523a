/* lgh_rows.h -- row-sharded operators and priors (rows.cu). */

#ifndef LGH_ROWS_H
#define LGH_ROWS_H

#include <vector>

#include "lgh_internal.h"

struct lgh_mat_s;
struct lgh_prior;

namespace lgh
{

/* The halo plan of one row-sharded operator on one rank: the local
 * operator (the Mat's Csr) multiplies an extended row-major block
 * [owned rows; ghost rows] whose ghost rows arrive from their owners in
 * one all-to-all per product, in owner order (ghosts are ascending global
 * rows and ranks own contiguous ranges, so the received bytes are the
 * ghost rows in place). */
struct RowsPlan
{
  lgh_rows_comm_t comm{};
  int64_t N = 0, row0 = 0, row1 = 0, nloc = 0, nghost = 0;
  std::vector<int64_t> send_rows;   /* rows sent to each peer            */
  std::vector<int64_t> recv_rows;   /* ghost rows received from each peer */
  DBuf<int64_t> sidx;               /* local send rows, peers in rank order */
  int64_t nsend = 0;
  DBuf<char> sbuf, xext;            /* packed send rows; extended block  */
  std::vector<size_t> sbytes, rbytes;
  long exchanges = 0;
  int64_t bytes_sent = 0;
  double seconds = 0.;
};

/* Workspace and the rank-local preconditioner of a row-sharded prior:
 * diag is Z restricted to the owned rows and columns (the block-Jacobi
 * block), on which the prior's multigrid hierarchy is built. */
struct RowsPrior
{
  Csr diag;
  int ld = 0;
  DBuf<double> X, R, P, Q, Z, T;    /* nloc x ld iterates                 */
  DBuf<double> part, sums;          /* column-sum partials and results    */
  DBuf<double> coef;                /* per-column alpha / beta (device)   */
  std::vector<double> h;            /* host mirror of the sums            */
  /* the global coarse correction (AMG type, hierarchies of two levels or
   * more): the coarse space is every rank's first-level aggregates (the
   * local prolongator P_r of the diagonal block's hierarchy), the coarse
   * operator A_c = P^T Z P of the whole Z (couplings across slabs
   * included), replicated on every rank with a hierarchy of its own.
   * coarse: 0 none (block Jacobi), 1 additive, 2 symmetric multiplicative */
  int coarse = 0;
  int64_t nc = 0, nc_loc = 0, coff = 0;
  Csr cA;
  Hierarchy *cmg = nullptr;
  DBuf<double> rc, ec;              /* nc x ld coarse blocks              */
};

/* the shard plan for rank `rank` of an explicit contiguous partition
 * (rank r owns [starts[r], starts[r + 1]); shard.cu) */
int shard_create_ranges (int64_t N, int nranks, int rank,
                         const int64_t *starts, const int64_t *rowptr,
                         const int32_t *colidx, lgh_shard_t **out);

/* the same communicator (rank, size, callbacks, context) */
bool rows_same_comm (const lgh_rows_comm_t &a, const lgh_rows_comm_t &b);

/* buf[0, count) summed over ranks (stream synchronised first) */
int rows_allreduce (const lgh_rows_comm_t &c, double *buf, size_t count,
                    cudaStream_t s);

/* Y = A X for a row-sharded Mat (the halo exchange, then the local
 * product): X holds the owned rows (ld ldx), Y the owned rows of A X */
template <typename T>
int rows_mult_block (lgh_mat_s *A, const T *X, int ldx, T *Y, int ldy, int w,
                     cudaStream_t s);

void rows_plan_free (RowsPlan *P);

/* the rank-local preconditioner of a row-sharded prior (diagonal block,
 * multigrid hierarchy for the AMG type) */
int rows_prior_setup (lgh_prior *p);
void rows_prior_free (RowsPrior *R);

/* Y = Z^{-1} (s_in .* X) .* s_out over the slabs: blocked PCG, FP64
 * iterates, block-Jacobi preconditioner, per-column tolerance rtol */
template <typename T>
int rows_zsolve (lgh_prior *p, int w, const T *X, int ldx, const double *s_in,
                 T *Y, int ldy, const double *s_out, double rtol);

} /* namespace lgh */

#endif /* LGH_ROWS_H */
