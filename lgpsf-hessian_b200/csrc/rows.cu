/* rows.cu -- a build over row slabs, one rank per GPU.
 *
 * The reference runs its whole pipeline on MPI row slabs (PETSc MPIAIJ /
 * MPIDENSE; docs/glr-woodbury-formulas.tex:76-98): MatMult scatters the
 * ghost entries of x before the local product, KSP's dot products are
 * all-reduced, and every Gram / Q^T F Q / U^T X is a local product plus
 * MPI_Allreduce (glr_common_impl.h:363, 487, 769, 851).  Here:
 *
 *   - a row-sharded operator (lgh_mat_create_rows) keeps the owned rows
 *     over local columns [owned; ghosts] and a halo plan; one product is
 *     one all-to-all of the ghost rows (received in place into the ghost
 *     rows of an extended block, since ghosts are ascending global rows
 *     and ranks own contiguous ranges) and the local strip / CSR product;
 *   - a row-sharded prior solves with blocked PCG whose dot products are
 *     all-reduced (two all-reduces of up to 2 w doubles per iteration);
 *     its preconditioner is the smoothed-aggregation V-cycle on the rank's
 *     diagonal block of Z (block Jacobi) with a global coarse correction
 *     (every rank's first-level aggregates, A_c = P^T Z P with the
 *     couplings across slabs, replicated), applied symmetric
 *     multiplicatively by default, or Jacobi.  Convergence is decided
 *     from the all-reduced sums only, so every rank takes the same
 *     iterations;
 *   - the in-process communicator runs ranks as threads of one process
 *     on one device: collectives meet on a host barrier with a time limit;
 *     no kernel ever waits for another rank.
 *
 * The exchange is the caller's (NCCL all_to_all_single / all_reduce over
 * NVLink in a torch.distributed job); the library synchronises its stream
 * before each callback, so the callback sees finished device data.
 */

#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <numeric>
#include <vector>

#include "lgh_internal.h"
#include "lgh_mg.h"
#include "lgh_objects.h"
#include "lgh_strip.h"

namespace lgh
{

namespace
{

int
egrid (int64_t total)
{
  int64_t g = (total + 255) / 256;
  g = std::max<int64_t> (1, std::min<int64_t> (g, (int64_t) num_sms () * 8));
  return (int) g;
}

/* E[i][c] = X[i][c] for c < w, 0 for w <= c < lde (the owned rows of the
 * extended block) */
template <typename T>
__global__ void
k_rows_own (int64_t n, int w, int lde, const T *__restrict__ X, int ldx,
            T *__restrict__ E)
{
  const int64_t total = n * lde;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / lde;
    const int c = (int) (e - i * lde);
    E[e] = c < w ? X[i * ldx + c] : T (0);
  }
}

/* buf[k][c] = X[idx[k]][c] (c < w; zero padding to lde): the rows one
 * rank sends, peers in rank order */
template <typename T>
__global__ void
k_rows_gather (int64_t count, int w, int lde, const int64_t *__restrict__ idx,
               const T *__restrict__ X, int ldx, T *__restrict__ buf)
{
  const int64_t total = count * lde;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t k = e / lde;
    const int c = (int) (e - k * lde);
    buf[e] = c < w ? X[idx[k] * ldx + c] : T (0);
  }
}

/* R[i][c] = s[i] X[i][c] (s null: 1) in FP64, zero padding to ld */
template <typename T>
__global__ void
k_rows_load (int64_t n, int w, int ld, const T *__restrict__ X, int ldx,
             const double *__restrict__ s, double *__restrict__ R)
{
  const int64_t total = n * ld;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / ld;
    const int c = (int) (e - i * ld);
    R[e] = c < w ? (s ? s[i] : 1.) * (double) X[i * ldx + c] : 0.;
  }
}

/* Y[i][c] = s[i] X[i][c] (s null: 1), c < w, converted to T */
template <typename T>
__global__ void
k_rows_store (int64_t n, int w, int ld, const double *__restrict__ X,
              const double *__restrict__ s, T *__restrict__ Y, int ldy)
{
  const int64_t total = n * w;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const int64_t i = e / w;
    const int c = (int) (e - i * w);
    Y[i * ldy + c] = (T) ((s ? s[i] : 1.) * X[i * ld + c]);
  }
}

/* part[b][c] (+ part[b][ld + c] for two pairs): block b's share of the
 * column sums of A .* B (and C .* D); rows strided over the grid, 8 row
 * lanes x 32 columns per CTA, fixed order (deterministic for a grid).
 * gridDim.y x 32 >= ld (ld = w rounded up to 4), so every c < ld is
 * written */
template <int PAIRS>
__global__ void __launch_bounds__ (256)
k_rows_dots (int64_t n, int w, int ld, const double *__restrict__ A,
             const double *__restrict__ B, const double *__restrict__ C,
             const double *__restrict__ D, double *__restrict__ part)
{
  __shared__ double sh[PAIRS][8][33];
  const int cl = threadIdx.x & 31, rl = threadIdx.x >> 5;
  const int c = blockIdx.y * 32 + cl;
  double s0 = 0., s1 = 0.;
  if (c < w) {
    for (int64_t i = (int64_t) blockIdx.x * 8 + rl; i < n;
         i += (int64_t) gridDim.x * 8) {
      const int64_t o = i * ld + c;
      s0 = fma (A[o], B[o], s0);
      if (PAIRS == 2) s1 = fma (C[o], D[o], s1);
    }
  }
  sh[0][rl][cl] = s0;
  if (PAIRS == 2) sh[PAIRS - 1][rl][cl] = s1;
  __syncthreads ();
  if (rl == 0 && c < ld) {            /* padding columns get zeros */
    double t0 = 0., t1 = 0.;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      t0 += sh[0][r][cl];
      if (PAIRS == 2) t1 += sh[PAIRS - 1][r][cl];
    }
    double *pb = part + (size_t) blockIdx.x * PAIRS * ld;
    pb[c] = t0;
    if (PAIRS == 2) pb[ld + c] = t1;
  }
}

/* out[c] = sum over the nb block partials, in block order */
__global__ void
k_rows_dots_fin (int nb, int cols, const double *__restrict__ part,
                 double *__restrict__ out)
{
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols;
       c += gridDim.x * blockDim.x) {
    double s = 0.;
    for (int b = 0; b < nb; b++) s += part[(size_t) b * cols + c];
    out[c] = s;
  }
}

/* x += alpha p, r -= alpha q (per-column alpha; zero for inactive) */
__global__ void
k_rows_step (int64_t n, int ld, const double *__restrict__ alpha,
             double *__restrict__ X, double *__restrict__ R,
             const double *__restrict__ P, const double *__restrict__ Q)
{
  const int64_t total = n * ld;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x) {
    const double a = alpha[e % ld];
    X[e] = fma (a, P[e], X[e]);
    R[e] = fma (-a, Q[e], R[e]);
  }
}

/* p = z + beta p */
__global__ void
k_rows_dir (int64_t n, int ld, const double *__restrict__ beta,
            const double *__restrict__ Z, double *__restrict__ P)
{
  const int64_t total = n * ld;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x)
    P[e] = fma (beta[e % ld], P[e], Z[e]);
}

/* out = a X + b Y (elementwise; out may alias X or Y) */
__global__ void
k_rows_axpby (int64_t total, double a, const double *X, double b,
              const double *Y, double *out)
{
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x)
    out[e] = a * X[e] + b * Y[e];
}

/* z = D^{-1} r (the Jacobi type of the rank-local preconditioner) */
__global__ void
k_rows_jacobi (int64_t n, int ld, const double *__restrict__ dinv,
               const double *__restrict__ R, double *__restrict__ Z)
{
  const int64_t total = n * ld;
  for (int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t) gridDim.x * blockDim.x)
    Z[e] = dinv[e / ld] * R[e];
}

} /* namespace */

bool
rows_same_comm (const lgh_rows_comm_t &a, const lgh_rows_comm_t &b)
{
  return a.rank == b.rank && a.size == b.size && a.allreduce == b.allreduce
         && a.alltoallv == b.alltoallv && a.ctx == b.ctx;
}

int
rows_allreduce (const lgh_rows_comm_t &c, double *buf, size_t count,
                cudaStream_t s)
{
  if (c.size <= 1 || count == 0) return 0;
  LGH_CUDA (cudaStreamSynchronize (s));
  LGH_CHECK (c.allreduce (buf, count, c.ctx) == 0, LGH_ERR_GPU,
             "row slabs: the all-reduce failed (rank %d of %d)", c.rank,
             c.size);
  return 0;
}

/* Xext = [X; ghost rows] with leading dimension lde: the owned rows are
 * copied in, the peers' send rows packed, one all-to-all drops the ghost
 * rows in place after the owned rows */
template <typename T>
static int
rows_halo (RowsPlan &P, const T *X, int ldx, int w, T **Xext, int *lde_out,
           cudaStream_t s)
{
  const int lde = round_ld (w);
  const size_t rowb = (size_t) lde * sizeof (T);
  LGH_TRY (P.xext.alloc ((size_t) (P.nloc + P.nghost) * rowb));
  T *E = (T *) P.xext.p;
  k_rows_own<T><<<egrid (P.nloc * lde), 256, 0, s>>> (P.nloc, w, lde, X, ldx, E);
  LGH_LAUNCH_CHECK ();
  if (P.comm.size > 1) {
    if (P.nsend > 0) {
      LGH_TRY (P.sbuf.alloc ((size_t) P.nsend * rowb));
      k_rows_gather<T><<<egrid (P.nsend * lde), 256, 0, s>>> (
          P.nsend, w, lde, P.sidx.p, X, ldx, (T *) P.sbuf.p);
      LGH_LAUNCH_CHECK ();
    }
    const int np = P.comm.size;
    P.sbytes.assign (np, 0);
    P.rbytes.assign (np, 0);
    size_t sent = 0;
    for (int q = 0; q < np; q++) {
      P.sbytes[q] = (size_t) P.send_rows[q] * rowb;
      P.rbytes[q] = (size_t) P.recv_rows[q] * rowb;
      sent += P.sbytes[q];
    }
    LGH_CUDA (cudaStreamSynchronize (s));
    const double t0 = wall ();
    const int rc = P.comm.alltoallv (P.sbuf.p, P.sbytes.data (),
                                     (char *) E + (size_t) P.nloc * rowb,
                                     P.rbytes.data (), P.comm.ctx);
    P.seconds += wall () - t0;
    LGH_CHECK (rc == 0, LGH_ERR_GPU,
               "row slabs: the halo exchange failed (rank %d of %d)",
               P.comm.rank, P.comm.size);
    P.exchanges++;
    P.bytes_sent += (int64_t) sent;
  }
  *Xext = E;
  *lde_out = lde;
  return 0;
}

template <typename T>
int
rows_mult_block (lgh_mat_s *A, const T *X, int ldx, T *Y, int ldy, int w,
                 cudaStream_t s)
{
  if (w == 0) return 0;
  T *E;
  int lde;
  LGH_TRY (rows_halo<T> (*A->rows, X, ldx, w, &E, &lde, s));
  if (w >= 8) {
    LGH_TRY (mat_prepare_block (A, w));
    return launch_strip_spmm<T> (A->strips, E, lde, Y, ldy, w, s);
  }
  return launch_spmm<T> (A->csr, E, lde, Y, ldy, w, s);
}

template int rows_mult_block<double> (lgh_mat_s *, const double *, int,
                                      double *, int, int, cudaStream_t);
template int rows_mult_block<float> (lgh_mat_s *, const float *, int, float *,
                                     int, int, cudaStream_t);

void
rows_plan_free (RowsPlan *P)
{
  delete P;
}

/* ---- the row-sharded prior ---------------------------------------------- */

/* one all-to-all of host int64 arrays through device buffers */
static int
rows_exchange_i64 (const lgh_rows_comm_t &c, const std::vector<int64_t> &send,
                   const std::vector<size_t> &scount,
                   std::vector<int64_t> &recv,
                   const std::vector<size_t> &rcount)
{
  const int np = c.size;
  std::vector<size_t> sb (np), rb (np);
  size_t rtot = 0;
  for (int p = 0; p < np; p++) {
    sb[p] = scount[p] * sizeof (int64_t);
    rb[p] = rcount[p] * sizeof (int64_t);
    rtot += rcount[p];
  }
  DBuf<int64_t> ds, dr;
  LGH_TRY (ds.alloc (std::max<size_t> (send.size (), 1)));
  LGH_TRY (dr.alloc (std::max<size_t> (rtot, 1)));
  if (!send.empty ())
    LGH_CUDA (cudaMemcpy (ds.p, send.data (), send.size () * sizeof (int64_t),
                          cudaMemcpyHostToDevice));
  LGH_CHECK (c.alltoallv (ds.p, sb.data (), dr.p, rb.data (), c.ctx) == 0,
             LGH_ERR_GPU, "row slabs: the plan exchange failed (rank %d of %d)",
             c.rank, c.size);
  recv.resize (rtot);
  if (rtot)
    LGH_CUDA (cudaMemcpy (recv.data (), dr.p, rtot * sizeof (int64_t),
                          cudaMemcpyDeviceToHost));
  return 0;
}

template <typename T>
static int
host_copy (std::vector<T> &h, const T *d, int64_t count)
{
  h.resize (count);
  if (count)
    LGH_CUDA (cudaMemcpy (h.data (), d, count * sizeof (T),
                          cudaMemcpyDeviceToHost));
  return 0;
}

static int64_t
pack_double (double v)
{
  int64_t b;
  memcpy (&b, &v, sizeof b);
  return b;
}

static double
unpack_double (int64_t b)
{
  double v;
  memcpy (&v, &b, sizeof v);
  return v;
}

/* The global coarse correction (RowsPrior): the global coarse numbering
 * (rank r's aggregates after those of ranks < r), the P rows of the Z
 * halo's ghost rows from their owners, this rank's rows of
 * A_c = P^T Z P, then every rank's rows to every rank and the coarse
 * hierarchy.  All ranks compute the same A_c and build the same
 * hierarchy on it. */
static int
rows_coarse_setup (lgh_prior *p, int mode)
{
  RowsPrior &W = *p->rows;
  Hierarchy *h = p->mg;
  W.coarse = 0;
  if (mode <= 0 || h == nullptr || h->lev.size () < 2) return 0;
  const RowsPlan &Zp = *p->Z->rows;
  const lgh_rows_comm_t &cm = Zp.comm;
  const int np = cm.size, me = cm.rank;
  cudaStream_t s = stream ();
  const Csr &Pd = h->lev[0].P;
  const int64_t nloc = Pd.n, ncl = h->lev[1].n;
  std::vector<int64_t> prp, zrp;
  std::vector<int32_t> pci, zci;
  std::vector<double> pva, zva;
  LGH_TRY (host_copy (prp, Pd.rowptr, nloc + 1));
  LGH_TRY (host_copy (pci, Pd.colidx, Pd.nnz));
  LGH_TRY (host_copy (pva, Pd.vals, Pd.nnz));
  const Csr &Zc = p->Z->csr;
  LGH_TRY (host_copy (zrp, Zc.rowptr, Zc.n + 1));
  LGH_TRY (host_copy (zci, Zc.colidx, Zc.nnz));
  LGH_TRY (host_copy (zva, Zc.vals, Zc.nnz));

  /* coarse offsets: each rank's count in its slot, summed */
  std::vector<double> cnt (np, 0.);
  cnt[me] = (double) ncl;
  {
    DBuf<double> d;
    LGH_TRY (d.alloc (np));
    LGH_CUDA (cudaMemcpy (d.p, cnt.data (), np * sizeof (double),
                          cudaMemcpyHostToDevice));
    LGH_TRY (rows_allreduce (cm, d.p, np, s));
    LGH_CUDA (cudaMemcpy (cnt.data (), d.p, np * sizeof (double),
                          cudaMemcpyDeviceToHost));
  }
  std::vector<int64_t> coff (np + 1, 0);
  for (int q = 0; q < np; q++) coff[q + 1] = coff[q] + (int64_t) llround (cnt[q]);
  const int64_t nc = coff[np], c0 = coff[me];
  LGH_CHECK (nc < (int64_t) INT32_MAX, LGH_ERR_ARG_OUTOFRANGE,
             "row slabs: coarse space of %lld rows", (long long) nc);

  /* the P rows of the Z halo's send rows, to the peers that hold them as
   * ghosts: per-row counts, then (global coarse column, value) pairs */
  std::vector<int64_t> sidx;
  LGH_TRY (host_copy (sidx, Zp.sidx.p, Zp.nsend));
  std::vector<int64_t> snnz, sent, gnnz, gent;
  std::vector<size_t> rs (np), rr (np), es (np, 0), er (np, 0);
  for (int q = 0, k = 0; q < np; q++) {
    rs[q] = (size_t) Zp.send_rows[q];
    rr[q] = (size_t) Zp.recv_rows[q];
    for (int64_t t = 0; t < Zp.send_rows[q]; t++, k++) {
      const int64_t i = sidx[k];
      snnz.push_back (prp[i + 1] - prp[i]);
      for (int64_t e = prp[i]; e < prp[i + 1]; e++) {
        sent.push_back (c0 + pci[e]);
        sent.push_back (pack_double (pva[e]));
      }
      es[q] += 2 * (size_t) (prp[i + 1] - prp[i]);
    }
  }
  LGH_TRY (rows_exchange_i64 (cm, snnz, rs, gnnz, rr));
  for (int q = 0, g = 0; q < np; q++)
    for (int64_t t = 0; t < Zp.recv_rows[q]; t++, g++) er[q] += 2 * (size_t) gnnz[g];
  LGH_TRY (rows_exchange_i64 (cm, sent, es, gent, er));
  std::vector<int64_t> grp (Zp.nghost + 1, 0);
  for (int64_t g = 0; g < Zp.nghost; g++) grp[g + 1] = grp[g] + gnnz[g];

  /* this rank's coarse rows: A_c[I, :] = sum_i P[i, I] (Z P)[i, :] */
  std::vector<int64_t> tp (ncl + 1, 0), ti (pci.size ());
  std::vector<double> tv (pci.size ());
  for (size_t e = 0; e < pci.size (); e++) tp[pci[e] + 1]++;
  for (int64_t I = 0; I < ncl; I++) tp[I + 1] += tp[I];
  {
    std::vector<int64_t> fill (tp.begin (), tp.end () - 1);
    for (int64_t i = 0; i < nloc; i++)
      for (int64_t e = prp[i]; e < prp[i + 1]; e++) {
        const int64_t at = fill[pci[e]]++;
        ti[at] = i;
        tv[at] = pva[e];
      }
  }
  std::vector<double> acc (nc, 0.);
  std::vector<char> mark (nc, 0);
  std::vector<int64_t> list, arp (ncl + 1, 0), aci;
  std::vector<double> ava;
  auto add = [&] (int64_t J, double v) {
    if (!mark[J]) { mark[J] = 1; list.push_back (J); }
    acc[J] += v;
  };
  for (int64_t I = 0; I < ncl; I++) {
    list.clear ();
    for (int64_t t = tp[I]; t < tp[I + 1]; t++) {
      const int64_t i = ti[t];
      for (int64_t k = zrp[i]; k < zrp[i + 1]; k++) {
        const int64_t c = zci[k];
        const double f = tv[t] * zva[k];
        if (c < nloc) {
          for (int64_t e = prp[c]; e < prp[c + 1]; e++)
            add (c0 + pci[e], f * pva[e]);
        } else {
          const int64_t g = c - nloc;
          for (int64_t e = grp[g]; e < grp[g + 1]; e++)
            add (gent[2 * e], f * unpack_double (gent[2 * e + 1]));
        }
      }
    }
    std::sort (list.begin (), list.end ());
    for (int64_t J : list) {
      aci.push_back (J);
      ava.push_back (acc[J]);
      acc[J] = 0.;
      mark[J] = 0;
    }
    arp[I + 1] = (int64_t) aci.size ();
  }

  /* every rank's rows to every rank */
  std::vector<int64_t> mynnz (ncl), myent;
  for (int64_t I = 0; I < ncl; I++) mynnz[I] = arp[I + 1] - arp[I];
  for (size_t e = 0; e < aci.size (); e++) {
    myent.push_back (aci[e]);
    myent.push_back (pack_double (ava[e]));
  }
  std::vector<int64_t> bnnz, bent, rnnz, rent;
  std::vector<size_t> ns (np, 0), nr (np, 0), xs (np, 0), xr (np, 0);
  for (int q = 0; q < np; q++) {
    if (q == me) continue;
    bnnz.insert (bnnz.end (), mynnz.begin (), mynnz.end ());
    bent.insert (bent.end (), myent.begin (), myent.end ());
    ns[q] = (size_t) ncl;
    nr[q] = (size_t) (coff[q + 1] - coff[q]);
    xs[q] = myent.size ();
  }
  LGH_TRY (rows_exchange_i64 (cm, bnnz, ns, rnnz, nr));
  {
    size_t k = 0;
    for (int q = 0; q < np; q++) {
      if (q == me) continue;
      for (size_t t = 0; t < nr[q]; t++, k++) xr[q] += 2 * (size_t) rnnz[k];
    }
  }
  LGH_TRY (rows_exchange_i64 (cm, bent, xs, rent, xr));
  std::vector<int64_t> crp (nc + 1, 0);
  std::vector<int32_t> cci;
  std::vector<double> cva;
  {
    size_t kr = 0, ke = 0;
    for (int q = 0; q < np; q++) {
      const int64_t rows_q = coff[q + 1] - coff[q];
      for (int64_t I = 0; I < rows_q; I++) {
        const int64_t gI = coff[q] + I;
        if (q == me) {
          for (int64_t e = arp[I]; e < arp[I + 1]; e++) {
            cci.push_back ((int32_t) aci[e]);
            cva.push_back (ava[e]);
          }
        } else {
          const int64_t m = rnnz[kr++];
          for (int64_t t = 0; t < m; t++, ke++) {
            cci.push_back ((int32_t) rent[2 * ke]);
            cva.push_back (unpack_double (rent[2 * ke + 1]));
          }
        }
        crp[gI + 1] = (int64_t) cci.size ();
      }
    }
  }
  Csr &A = W.cA;
  A.n = nc;
  A.nnz = (int64_t) cci.size ();
  LGH_TRY (dalloc ((void **) &A.rowptr, (size_t) (nc + 1) * sizeof (int64_t)));
  LGH_TRY (dalloc ((void **) &A.colidx, (size_t) A.nnz * sizeof (int32_t) + 16));
  LGH_TRY (dalloc ((void **) &A.vals, (size_t) A.nnz * sizeof (double) + 16));
  LGH_CUDA (cudaMemcpy (A.rowptr, crp.data (), (nc + 1) * sizeof (int64_t),
                        cudaMemcpyHostToDevice));
  LGH_CUDA (cudaMemcpy (A.colidx, cci.data (), A.nnz * sizeof (int32_t),
                        cudaMemcpyHostToDevice));
  LGH_CUDA (cudaMemcpy (A.vals, cva.data (), A.nnz * sizeof (double),
                        cudaMemcpyHostToDevice));
  LGH_TRY (csr_finish (A));
  const lgh_prior_mat_opts_t &o = p->mopts;
  LGH_TRY (mg_build (A, o.tile, o.smoother_top, o.nu_force > 0 ? o.nu_force : 2,
                     &W.cmg));
  W.coarse = mode;
  W.nc = nc;
  W.nc_loc = ncl;
  W.coff = c0;
  return 0;
}

/* diag = Z restricted to the owned rows and columns (local columns below
 * nloc), and its multigrid hierarchy for the AMG type */
int
rows_prior_setup (lgh_prior *p)
{
  const Csr &A = p->Z->csr;
  const int64_t n = A.n, nnz = A.nnz;
  std::vector<int64_t> rp (n + 1);
  std::vector<int32_t> ci (nnz);
  std::vector<double> va (nnz);
  LGH_CUDA (cudaMemcpy (rp.data (), A.rowptr, (n + 1) * sizeof (int64_t),
                        cudaMemcpyDeviceToHost));
  if (nnz) {
    LGH_CUDA (cudaMemcpy (ci.data (), A.colidx, nnz * sizeof (int32_t),
                          cudaMemcpyDeviceToHost));
    LGH_CUDA (cudaMemcpy (va.data (), A.vals, nnz * sizeof (double),
                          cudaMemcpyDeviceToHost));
  }
  std::vector<int64_t> drp (n + 1, 0);
  std::vector<int32_t> dci;
  std::vector<double> dva;
  dci.reserve (nnz);
  dva.reserve (nnz);
  for (int64_t i = 0; i < n; i++) {
    for (int64_t k = rp[i]; k < rp[i + 1]; k++)
      if (ci[k] < n) {
        dci.push_back (ci[k]);
        dva.push_back (va[k]);
      }
    drp[i + 1] = (int64_t) dci.size ();
  }
  RowsPrior *R = p->rows;
  Csr &D = R->diag;
  D.n = n;
  D.nnz = (int64_t) dci.size ();
  LGH_TRY (dalloc ((void **) &D.rowptr, (size_t) (n + 1) * sizeof (int64_t)));
  LGH_TRY (dalloc ((void **) &D.colidx, (size_t) D.nnz * sizeof (int32_t) + 16));
  LGH_TRY (dalloc ((void **) &D.vals, (size_t) D.nnz * sizeof (double) + 16));
  LGH_CUDA (cudaMemcpy (D.rowptr, drp.data (), (n + 1) * sizeof (int64_t),
                        cudaMemcpyHostToDevice));
  if (D.nnz) {
    LGH_CUDA (cudaMemcpy (D.colidx, dci.data (), D.nnz * sizeof (int32_t),
                          cudaMemcpyHostToDevice));
    LGH_CUDA (cudaMemcpy (D.vals, dva.data (), D.nnz * sizeof (double),
                          cudaMemcpyHostToDevice));
  }
  LGH_TRY (csr_finish (D));
  if (p->pc_type == LGH_PC_AMG) {
    const lgh_prior_mat_opts_t &o = p->mopts;
    const int nu = o.nu_force > 0 ? o.nu_force : 2;
    LGH_TRY (mg_build (D, o.tile, o.smoother_top, nu, &p->mg));
    /* LGH_ROWS_COARSE: 0 block Jacobi alone, 1 additive, 2 symmetric
     * multiplicative coarse correction (default) */
    const char *env = getenv ("LGH_ROWS_COARSE");
    LGH_TRY (rows_coarse_setup (p, env ? atoi (env) : 2));
  }
  return 0;
}

void
rows_prior_free (RowsPrior *R)
{
  if (!R) return;
  if (R->cmg) mg_destroy (R->cmg);     /* borrows cA's arrays */
  csr_free (R->cA);
  csr_free (R->diag);
  delete R;
}

template <typename T>
int
rows_zsolve (lgh_prior *p, int w, const T *X, int ldx, const double *s_in,
             T *Y, int ldy, const double *s_out, double rtol)
{
  if (w == 0) return 0;
  cudaStream_t s = stream ();
  RowsPrior &W = *p->rows;
  const lgh_rows_comm_t &cm = p->Z->rows->comm;
  const int64_t n = p->n;
  const int ld = round_ld (w);
  const size_t nn = (size_t) n * ld;
  const double t0 = wall ();
  LGH_TRY (W.X.alloc (nn));
  LGH_TRY (W.R.alloc (nn));
  LGH_TRY (W.P.alloc (nn));
  LGH_TRY (W.Q.alloc (nn));
  LGH_TRY (W.Z.alloc (nn));
  const int gx = (int) std::max<int64_t> (
      1, std::min<int64_t> ((n + 7) / 8, 2 * (int64_t) num_sms ()));
  const int gy = (w + 31) / 32;
  LGH_TRY (W.part.alloc ((size_t) gx * 2 * ld));
  LGH_TRY (W.sums.alloc (2 * (size_t) ld));
  LGH_TRY (W.coef.alloc (2 * (size_t) ld));
  W.h.assign (2 * (size_t) ld, 0.);

  /* h[0, ld) (and h[ld, 2 ld)) = the all-reduced column sums of A .* B
   * (and C .* D) */
  auto colsums = [&] (int pairs, const double *A, const double *B,
                      const double *C, const double *D) -> int {
    const dim3 g (gx, gy);
    if (pairs == 2)
      k_rows_dots<2><<<g, 256, 0, s>>> (n, w, ld, A, B, C, D, W.part.p);
    else
      k_rows_dots<1><<<g, 256, 0, s>>> (n, w, ld, A, B, nullptr, nullptr,
                                        W.part.p);
    LGH_LAUNCH_CHECK ();
    const int cols = pairs * ld;
    k_rows_dots_fin<<<(cols + 255) / 256, 256, 0, s>>> (gx, cols, W.part.p,
                                                        W.sums.p);
    LGH_LAUNCH_CHECK ();
    LGH_TRY (rows_allreduce (cm, W.sums.p, cols, s));
    LGH_CUDA (cudaMemcpyAsync (W.h.data (), W.sums.p, cols * sizeof (double),
                               cudaMemcpyDeviceToHost, s));
    LGH_CUDA (cudaStreamSynchronize (s));
    return 0;
  };
  if (W.coarse) {
    LGH_TRY (W.rc.alloc ((size_t) W.nc * ld));
    LGH_TRY (W.ec.alloc ((size_t) W.nc * ld));
    if (W.coarse == 2) LGH_TRY (W.T.alloc (nn));
  }
  /* t = r - Z z (the symmetric multiplicative form's residuals) */
  auto resid = [&] (const double *z) -> int {
    LGH_TRY (rows_mult_block<double> (p->Z, z, ld, W.T.p, ld, w, s));
    k_rows_axpby<<<egrid ((int64_t) nn), 256, 0, s>>> ((int64_t) nn, 1., W.R.p,
                                                        -1., W.T.p, W.T.p);
    LGH_LAUNCH_CHECK ();
    return 0;
  };
  /* z += P V_c (P^T t): the coarse rows of every rank summed into one
   * zero-filled nc-row block (exact: the other slots add zeros) */
  auto coarse = [&] (const double *t) -> int {
    const MgLevel &l0 = p->mg->lev[0];
    LGH_CUDA (cudaMemsetAsync (W.rc.p, 0, (size_t) W.nc * ld * sizeof (double), s));
    LGH_TRY (launch_spmm<double> (l0.R, t, ld, W.rc.p + (size_t) W.coff * ld,
                                  ld, w, s));
    LGH_TRY (rows_allreduce (cm, W.rc.p, (size_t) W.nc * ld, s));
    LGH_TRY (mg_vcycle<double> (W.cmg, W.rc.p, W.ec.p, ld, w, s));
    return launch_spmm_mode<double> (l0.P, W.ec.p + (size_t) W.coff * ld, ld,
                                     W.Z.p, ld, w, 1, nullptr, 0, s);
  };
  auto precond = [&] () -> int {
    if (!p->mg) {
      k_rows_jacobi<<<egrid ((int64_t) nn), 256, 0, s>>> (n, ld, W.diag.dinv,
                                                           W.R.p, W.Z.p);
      LGH_LAUNCH_CHECK ();
      return 0;
    }
    LGH_TRY (mg_vcycle<double> (p->mg, W.R.p, W.Z.p, ld, w, s));
    if (W.coarse == 1) return coarse (W.R.p);
    if (W.coarse == 2) {
      /* z1 = V r; z2 = z1 + P V_c P^T (r - Z z1); z = z2 + V (r - Z z2),
       * the last V-cycle's output in Q (free between products) */
      LGH_TRY (resid (W.Z.p));
      LGH_TRY (coarse (W.T.p));
      LGH_TRY (resid (W.Z.p));
      LGH_TRY (mg_vcycle<double> (p->mg, W.T.p, W.Q.p, ld, w, s));
      k_rows_axpby<<<egrid ((int64_t) nn), 256, 0, s>>> ((int64_t) nn, 1.,
                                                          W.Z.p, 1., W.Q.p,
                                                          W.Z.p);
      LGH_LAUNCH_CHECK ();
    }
    return 0;
  };

  k_rows_load<T><<<egrid ((int64_t) nn), 256, 0, s>>> (n, w, ld, X, ldx, s_in,
                                                        W.R.p);
  LGH_LAUNCH_CHECK ();
  /* zero padding columns stay zero through every pass */
  LGH_CUDA (cudaMemsetAsync (W.X.p, 0, nn * sizeof (double), s));
  LGH_CUDA (cudaMemsetAsync (W.Z.p, 0, nn * sizeof (double), s));
  LGH_CUDA (cudaMemsetAsync (W.Q.p, 0, nn * sizeof (double), s));
  LGH_TRY (precond ());
  LGH_TRY (colsums (2, W.R.p, W.Z.p, W.Z.p, W.Z.p));
  std::vector<double> rz (w), n0 (w), alpha (ld, 0.), beta (ld, 0.);
  std::vector<int> act (w, 0), its (w, 0);
  int nact = 0;
  for (int c = 0; c < w; c++) {
    rz[c] = W.h[c];
    n0[c] = sqrt (W.h[ld + c]);
    act[c] = W.h[ld + c] > 0. ? 1 : 0;
    nact += act[c];
  }
  LGH_CUDA (cudaMemcpyAsync (W.P.p, W.Z.p, nn * sizeof (double),
                             cudaMemcpyDeviceToDevice, s));
  int iters = 0;
  for (int it = 0; it < p->zcfg.maxit && nact > 0; it++) {
    LGH_TRY (rows_mult_block<double> (p->Z, W.P.p, ld, W.Q.p, ld, w, s));
    LGH_TRY (colsums (1, W.P.p, W.Q.p, nullptr, nullptr));
    for (int c = 0; c < w; c++) {
      alpha[c] = 0.;
      if (!act[c]) continue;
      const double pq = W.h[c];
      if (pq != 0. && isfinite (pq)) {
        alpha[c] = rz[c] / pq;
      } else {
        act[c] = 0;
        its[c] = it;
        nact--;
      }
    }
    LGH_CUDA (cudaMemcpyAsync (W.coef.p, alpha.data (), ld * sizeof (double),
                               cudaMemcpyHostToDevice, s));
    k_rows_step<<<egrid ((int64_t) nn), 256, 0, s>>> (n, ld, W.coef.p, W.X.p,
                                                       W.R.p, W.P.p, W.Q.p);
    LGH_LAUNCH_CHECK ();
    LGH_TRY (precond ());
    LGH_TRY (colsums (2, W.R.p, W.Z.p, W.Z.p, W.Z.p));
    for (int c = 0; c < w; c++) {
      beta[c] = 0.;
      if (!act[c]) continue;
      const double srz = W.h[c], szz = W.h[ld + c];
      const double b = rz[c] != 0. ? srz / rz[c] : 0.;
      rz[c] = srz;
      if (sqrt (szz) <= rtol * n0[c] || srz == 0.) {
        act[c] = 0;
        its[c] = it + 1;
        nact--;
      } else {
        beta[c] = b;
      }
    }
    LGH_CUDA (cudaMemcpyAsync (W.coef.p + ld, beta.data (), ld * sizeof (double),
                               cudaMemcpyHostToDevice, s));
    k_rows_dir<<<egrid ((int64_t) nn), 256, 0, s>>> (n, ld, W.coef.p + ld,
                                                      W.Z.p, W.P.p);
    LGH_LAUNCH_CHECK ();
    iters = it + 1;
  }
  long col_its = 0;
  for (int c = 0; c < w; c++) col_its += act[c] ? iters : its[c];
  k_rows_store<T><<<egrid (n * w), 256, 0, s>>> (n, w, ld, W.X.p, s_out, Y, ldy);
  LGH_LAUNCH_CHECK ();
  LGH_CUDA (cudaStreamSynchronize (s));
  ZsolveStats &st = p->stats;
  st.calls++;
  st.block_iters += iters;
  st.col_iters += col_its;
  st.cols += w;
  st.seconds += wall () - t0;
  st.last_maxit_hit = nact > 0 ? 1 : 0;
  return 0;
}

template int rows_zsolve<double> (lgh_prior *, int, const double *, int,
                                  const double *, double *, int,
                                  const double *, double);
template int rows_zsolve<float> (lgh_prior *, int, const float *, int,
                                 const double *, float *, int, const double *,
                                 double);

} /* namespace lgh */

/* ---- the C ABI ----------------------------------------------------------- */

using namespace lgh;

namespace
{

/* all ranks learn whether any rank failed a local step (one all-reduce of
 * a flag), so that no rank is left waiting in a later collective */
int
rows_agree (const lgh_rows_comm_t &c, int local_rc, const char *who)
{
  DBuf<double> f;
  LGH_TRY (f.alloc (1));
  const double v = local_rc ? 1. : 0.;
  LGH_CUDA (cudaMemcpy (f.p, &v, sizeof (double), cudaMemcpyHostToDevice));
  LGH_TRY (rows_allreduce (c, f.p, 1, stream ()));
  double sum = 0.;
  LGH_CUDA (cudaMemcpy (&sum, f.p, sizeof (double), cudaMemcpyDeviceToHost));
  if (local_rc) return local_rc;
  LGH_CHECK (sum == 0., LGH_ERR_ARG_WRONG, "%s: %g other rank(s) failed", who,
             sum);
  return 0;
}

} /* namespace */

extern "C" {

int
lgh_mat_create_rows (int64_t N, const lgh_rows_comm_t *comm, int64_t row0,
                     int64_t nrows, const int64_t *rowptr,
                     const int32_t *colidx, const double *vals, lgh_Mat *out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (comm && rowptr && out, LGH_ERR_ARG_NULL,
             "lgh_mat_create_rows: NULL argument");
  LGH_CHECK (comm->size >= 1 && comm->rank >= 0 && comm->rank < comm->size
             && comm->allreduce && comm->alltoallv, LGH_ERR_ARG_WRONG,
             "lgh_mat_create_rows: communicator (rank %d of %d)", comm->rank,
             comm->size);
  const lgh_rows_comm_t &cm = *comm;
  const int np = cm.size, me = cm.rank;
  const int64_t nloc = nrows, row1 = row0 + nrows;

  /* every rank's rows: one all-reduce of the (first row, count) slots */
  std::vector<int64_t> starts (np + 1, 0);
  int rc = 0;
  {
    std::vector<double> sl (2 * np, 0.);
    sl[2 * me] = (double) row0;
    sl[2 * me + 1] = (double) nrows;
    DBuf<double> d;
    LGH_TRY (d.alloc (2 * np));
    LGH_CUDA (cudaMemcpy (d.p, sl.data (), 2 * np * sizeof (double),
                          cudaMemcpyHostToDevice));
    LGH_TRY (rows_allreduce (cm, d.p, 2 * np, stream ()));
    LGH_CUDA (cudaMemcpy (sl.data (), d.p, 2 * np * sizeof (double),
                          cudaMemcpyDeviceToHost));
    for (int q = 0; q < np && !rc; q++) {
      const int64_t a = (int64_t) sl[2 * q], m = (int64_t) sl[2 * q + 1];
      if (a != starts[q] || m < 0)
        rc = set_error (LGH_ERR_ARG_WRONG,
                        "lgh_mat_create_rows: rank %d's rows start at %lld, "
                        "not %lld (ranks own contiguous rows in rank order)",
                        q, (long long) a, (long long) starts[q]);
      starts[q + 1] = a + m;
    }
    if (!rc && starts[np] != N)
      rc = set_error (LGH_ERR_ARG_WRONG,
                      "lgh_mat_create_rows: the ranks' rows cover %lld of "
                      "%lld", (long long) starts[np], (long long) N);
  }

  /* local checks and the plan; every rank then agrees before exchanging */
  if (rc) {
  } else if (N < 1 || N >= (int64_t) INT32_MAX || nloc < 1)
    rc = set_error (LGH_ERR_ARG_OUTOFRANGE,
                    "lgh_mat_create_rows: N %lld, %lld rows on rank %d",
                    (long long) N, (long long) nloc, me);
  else if (rowptr[0] != 0 || rowptr[nloc] < 0
           || (rowptr[nloc] > 0 && (!colidx || !vals)))
    rc = set_error (LGH_ERR_ARG_WRONG,
                    "lgh_mat_create_rows: rowptr[0] must be 0 and the "
                    "arrays non-null");
  lgh_shard_t *sh = nullptr;
  if (!rc)
    rc = shard_create_ranges (N, np, me, starts.data (), rowptr, colidx, &sh);
  struct Guard
  {
    lgh_shard_t *s;
    ~Guard () { if (s) lgh_shard_destroy (s); }
  } guard{ sh };
  LGH_TRY (rows_agree (cm, rc, "lgh_mat_create_rows"));

  const int64_t *grows = nullptr, *gcount = nullptr;
  int64_t nghost = 0;
  LGH_TRY (lgh_shard_info (sh, nullptr, nullptr, &nghost));
  LGH_TRY (lgh_shard_ghosts (sh, &grows, &gcount));
  const int32_t *lcol = nullptr;
  LGH_TRY (lgh_shard_local_colidx (sh, &lcol));

  /* how many rows each peer needs from this rank, then which */
  std::vector<int64_t> cnt_send, cnt_recv;
  for (int p = 0; p < np; p++)
    if (p != me) cnt_send.push_back (gcount[p]);
  std::vector<size_t> c1 (np, 1);
  c1[me] = 0;
  LGH_TRY (rows_exchange_i64 (cm, cnt_send, c1, cnt_recv, c1));
  std::vector<int64_t> need_by (np, 0);
  for (int p = 0, k = 0; p < np; p++)
    if (p != me) need_by[p] = cnt_recv[k++];
  std::vector<int64_t> ghosts (grows, grows + nghost), req;
  std::vector<size_t> sc (np), rcn (np);
  for (int p = 0; p < np; p++) {
    sc[p] = (size_t) gcount[p];
    rcn[p] = (size_t) need_by[p];
  }
  LGH_TRY (rows_exchange_i64 (cm, ghosts, sc, req, rcn));
  rc = 0;
  size_t off = 0;
  for (int p = 0; p < np && !rc; p++) {
    if (p != me && need_by[p] > 0)
      rc = lgh_shard_set_sends (sh, p, need_by[p], req.data () + off);
    off += (size_t) need_by[p];
  }
  LGH_TRY (rows_agree (cm, rc, "lgh_mat_create_rows"));
  std::vector<int64_t> sidx;
  for (int p = 0; p < np; p++) {
    int64_t n_p = 0;
    const int64_t *lr = nullptr;
    LGH_TRY (lgh_shard_sends (sh, p, &n_p, &lr));
    sidx.insert (sidx.end (), lr, lr + n_p);
  }

  /* the local operator: rows sorted by local column (the strip form's
   * merge and the multigrid set-up take sorted rows) */
  const int64_t nnz = rowptr[nloc];
  std::vector<int32_t> lc (nnz);
  std::vector<double> lv (nnz);
  {
    std::vector<int64_t> ord;
    for (int64_t i = 0; i < nloc; i++) {
      const int64_t a = rowptr[i], b = rowptr[i + 1];
      ord.resize (b - a);
      std::iota (ord.begin (), ord.end (), a);
      std::sort (ord.begin (), ord.end (),
                 [&] (int64_t x, int64_t y) { return lcol[x] < lcol[y]; });
      for (int64_t k = a; k < b; k++) {
        lc[k] = lcol[ord[k - a]];
        lv[k] = vals[ord[k - a]];
      }
    }
  }
  lgh_mat_s *A = new lgh_mat_s ();
  A->kind = 0;
  Csr &C = A->csr;
  C.n = nloc;
  C.ncols = nloc + nghost;
  C.nnz = nnz;
  rc = dalloc ((void **) &C.rowptr, (size_t) (nloc + 1) * sizeof (int64_t));
  if (!rc) rc = dalloc ((void **) &C.colidx, (size_t) nnz * sizeof (int32_t) + 16);
  if (!rc) rc = dalloc ((void **) &C.vals, (size_t) nnz * sizeof (double) + 16);
  if (!rc && cudaMemcpy (C.rowptr, rowptr, (nloc + 1) * sizeof (int64_t),
                         cudaMemcpyHostToDevice) != cudaSuccess)
    rc = set_error (LGH_ERR_GPU, "lgh_mat_create_rows: copy");
  if (!rc && nnz
      && (cudaMemcpy (C.colidx, lc.data (), nnz * sizeof (int32_t),
                      cudaMemcpyHostToDevice) != cudaSuccess
          || cudaMemcpy (C.vals, lv.data (), nnz * sizeof (double),
                         cudaMemcpyHostToDevice) != cudaSuccess))
    rc = set_error (LGH_ERR_GPU, "lgh_mat_create_rows: copy");
  if (!rc) rc = csr_finish (C);
  RowsPlan *P = nullptr;
  if (!rc) {
    P = new RowsPlan ();
    P->comm = cm;
    P->N = N;
    P->row0 = row0;
    P->row1 = row1;
    P->nloc = nloc;
    P->nghost = nghost;
    P->send_rows = need_by;
    P->recv_rows.assign (gcount, gcount + np);
    P->nsend = (int64_t) sidx.size ();
    rc = P->sidx.alloc (std::max<size_t> (sidx.size (), 1));
    if (!rc && !sidx.empty ()
        && cudaMemcpy (P->sidx.p, sidx.data (), sidx.size () * sizeof (int64_t),
                       cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "lgh_mat_create_rows: copy");
  }
  if (rc) {
    delete P;
    csr_free (C);
    delete A;
    return rc;
  }
  A->rows = P;
  *out = A;
  return 0;
}

int
lgh_mat_rows_info (lgh_Mat A, int64_t *row0, int64_t *row1, int64_t *nghost)
{
  LGH_CHECK (A, LGH_ERR_ARG_NULL, "lgh_mat_rows_info: NULL Mat");
  const RowsPlan *P = A->rows;
  if (row0) *row0 = P ? P->row0 : 0;
  if (row1) *row1 = P ? P->row1 : (A->kind == 0 ? A->csr.n : A->nrows);
  if (nghost) *nghost = P ? P->nghost : 0;
  return 0;
}

int
lgh_mat_rows_traffic (lgh_Mat A, long *exchanges, int64_t *bytes_sent,
                      double *seconds)
{
  LGH_CHECK (A, LGH_ERR_ARG_NULL, "lgh_mat_rows_traffic: NULL Mat");
  const RowsPlan *P = A->rows;
  if (exchanges) *exchanges = P ? P->exchanges : 0;
  if (bytes_sent) *bytes_sent = P ? P->bytes_sent : 0;
  if (seconds) *seconds = P ? P->seconds : 0.;
  return 0;
}

} /* extern "C" */
