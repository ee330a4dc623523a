/* persist.cu -- saving and restoring a built GLR object.
 *
 * A serving process that restarts, or a second process that serves the
 * same model, should not pay for the build again: the object's state is
 * the treated spectrum, the raw spectrum, U (N x kept) and, for further
 * incremental extension, the sketch basis Q (N x ell) with the raw
 * projection A = Q^T F Q (ell x ell).  The reference keeps these only in
 * memory (struct lgh_glr, glr_common_impl.h:252-278); this file format is
 * this library's own.
 *
 * Layout (little-endian, this library's structs):
 *   "LGHGLR01", int64 N, int32 kept, int32 ell (0: no extension state),
 *   int32 corrected, double floor, lgh_glr_opts_t, lgh_exec_opts_t,
 *   lam[kept], lam_raw[kept], U row by row (N x kept), then if ell > 0
 *   Q row by row (N x ell, FP64) and A (ell x ell, column-major),
 *   and a 64-bit FNV-1a checksum of everything before it.
 */

#include <stdio.h>
#include <string.h>

#include <vector>

#include "lgh_internal.h"
#include "lgh_objects.h"

namespace lgh
{

namespace
{

struct Sink
{
  FILE *f = nullptr;
  uint64_t h = 1469598103934665603ULL;
  bool ok = true;
  void put (const void *p, size_t n)
  {
    const unsigned char *b = (const unsigned char *) p;
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ULL; }
    if (ok && n && fwrite (p, 1, n, f) != n) ok = false;
  }
};

struct Source
{
  FILE *f = nullptr;
  uint64_t h = 1469598103934665603ULL;
  bool ok = true;
  void get (void *p, size_t n)
  {
    if (ok && n && fread (p, 1, n, f) != n) ok = false;
    if (!ok) return;
    const unsigned char *b = (const unsigned char *) p;
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ULL; }
  }
};

const char MAGIC[8] = { 'L', 'G', 'H', 'G', 'L', 'R', '0', '1' };

/* device row-major (ld) -> host, w columns, in row slabs */
int
put_rows (Sink &o, const double *d, int64_t n, int w, int ld)
{
  const int64_t slab = std::max<int64_t> (1, (64 << 20) / (8 * std::max (w, 1)));
  std::vector<double> h ((size_t) std::min (n, slab) * w);
  for (int64_t r0 = 0; r0 < n; r0 += slab) {
    const int64_t nr = std::min (slab, n - r0);
    LGH_CUDA (cudaMemcpy2D (h.data (), (size_t) w * 8, d + r0 * ld, (size_t) ld * 8,
                            (size_t) w * 8, nr, cudaMemcpyDeviceToHost));
    o.put (h.data (), (size_t) nr * w * 8);
  }
  return 0;
}

int
get_rows (Source &in, double *d, int64_t n, int w, int ld)
{
  const int64_t slab = std::max<int64_t> (1, (64 << 20) / (8 * std::max (w, 1)));
  std::vector<double> h ((size_t) std::min (n, slab) * w);
  for (int64_t r0 = 0; r0 < n && in.ok; r0 += slab) {
    const int64_t nr = std::min (slab, n - r0);
    in.get (h.data (), (size_t) nr * w * 8);
    if (!in.ok) break;
    LGH_CUDA (cudaMemcpy2D (d + r0 * ld, (size_t) ld * 8, h.data (), (size_t) w * 8,
                            (size_t) w * 8, nr, cudaMemcpyHostToDevice));
  }
  return 0;
}

} /* namespace */

} /* namespace lgh */

using namespace lgh;

extern "C" {

int
lgh_glr_save (const lgh_glr_t *g, const char *path, int with_extension)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (g && path, LGH_ERR_ARG_NULL, "lgh_glr_save: NULL argument");
  LGH_CHECK (!g->rows, LGH_ERR_SUP, "lgh_glr_save: not on a row-sharded object");
  LGH_CUDA (cudaDeviceSynchronize ());
  const int has_q = (g->Q.p != nullptr || g->Q32.p != nullptr) && g->ell > 0;
  LGH_CHECK (!with_extension || has_q, LGH_ERR_ARG_WRONGSTATE,
             "lgh_glr_save: the object keeps no extension state (replicated "
             "backend, or loaded without it)");
  Sink o;
  o.f = fopen (path, "wb");
  LGH_CHECK (o.f != nullptr, LGH_ERR_ARG_WRONG, "lgh_glr_save: cannot open %s",
             path);
  const int64_t n = g->n;
  const int32_t kept = g->kept, ell = with_extension ? g->ell : 0;
  const int32_t corr = g->corrected;
  int rc = 0;
  o.put (MAGIC, 8);
  o.put (&n, 8);
  o.put (&kept, 4);
  o.put (&ell, 4);
  o.put (&corr, 4);
  o.put (&g->floor, 8);
  o.put (&g->opts, sizeof (g->opts));
  o.put (&g->exec, sizeof (g->exec));
  o.put (g->lam_h.data (), (size_t) kept * 8);
  std::vector<double> lraw (kept);
  if (kept > 0 && g->lraw_d.p)
    rc = cudaMemcpy (lraw.data (), g->lraw_d.p, (size_t) kept * 8,
                     cudaMemcpyDeviceToHost) == cudaSuccess ? 0
         : set_error (LGH_ERR_GPU, "lgh_glr_save: copy");
  o.put (lraw.data (), (size_t) kept * 8);
  if (!rc && kept > 0) rc = put_rows (o, g->U.p, n, kept, g->ldu);
  if (!rc && ell > 0) {
    if (g->Q.p) {
      rc = put_rows (o, g->Q.p, n, ell, g->ldq);
    } else {
      DBuf<double> q;
      rc = q.alloc ((size_t) n * g->ldq);
      if (!rc) rc = launch_f32_to_f64 (n, ell, g->Q32.p, g->ldq, q.p, g->ldq, stream ());
      if (!rc) rc = put_rows (o, q.p, n, ell, g->ldq);
    }
    std::vector<double> A ((size_t) ell * ell);
    if (!rc && cudaMemcpy (A.data (), g->A.p, A.size () * 8,
                           cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = set_error (LGH_ERR_GPU, "lgh_glr_save: copy");
    o.put (A.data (), A.size () * 8);
  }
  const uint64_t sum = o.h;
  if (!rc && o.ok && fwrite (&sum, 1, 8, o.f) != 8) o.ok = false;
  if (fclose (o.f) != 0) o.ok = false;
  if (rc) return rc;
  LGH_CHECK (o.ok, LGH_ERR_ARG_WRONG, "lgh_glr_save: write to %s failed", path);
  return 0;
}

int
lgh_glr_load (lgh_Mat B, lgh_prior_t *prior, const char *path,
              lgh_glr_t **out)
{
  LGH_TRY (ensure_init ());
  LGH_CHECK (B && prior && path && out, LGH_ERR_ARG_NULL,
             "lgh_glr_load: NULL argument");
  LGH_CHECK (B->kind == 0 && B->csr.n == prior->n, LGH_ERR_ARG_SIZ,
             "lgh_glr_load: B and prior sizes differ");
  LGH_CHECK (!B->rows && !prior->rows, LGH_ERR_SUP,
             "lgh_glr_load: not onto row-sharded operators");
  Source in;
  in.f = fopen (path, "rb");
  LGH_CHECK (in.f != nullptr, LGH_ERR_ARG_WRONG, "lgh_glr_load: cannot open %s",
             path);
  char magic[8];
  int64_t n = 0;
  int32_t kept = 0, ell = 0, corr = 0;
  double floor = 0.;
  lgh_glr_opts_t opts;
  lgh_exec_opts_t exec;
  in.get (magic, 8);
  in.get (&n, 8);
  in.get (&kept, 4);
  in.get (&ell, 4);
  in.get (&corr, 4);
  in.get (&floor, 8);
  in.get (&opts, sizeof (opts));
  in.get (&exec, sizeof (exec));
  const int prec = exec.precision;
  int rc = 0;
  if (!in.ok || memcmp (magic, MAGIC, 8) != 0)
    rc = set_error (LGH_ERR_ARG_WRONG, "lgh_glr_load: %s is not a saved GLR object",
                    path);
  else if (n != B->csr.n)
    rc = set_error (LGH_ERR_ARG_SIZ, "lgh_glr_load: saved N %lld, operator N %lld",
                    (long long) n, (long long) B->csr.n);
  else if (kept < 0 || ell < 0 || ell > 2048 || kept > 2048
           || (prec != LGH_PREC_FP64 && prec != LGH_PREC_MIXED))
    rc = set_error (LGH_ERR_ARG_WRONG, "lgh_glr_load: corrupt header in %s", path);
  lgh_glr_t *g = nullptr;
  if (!rc) {
    g = new lgh_glr_t ();
    g->n = n;
    g->opts = opts;
    g->exec = exec;
    g->corrected = corr;
    g->floor = floor;
    g->B = B;
    B->refs++;
    g->prior = prior;
    prior_ref (prior);
    g->kept = kept;
    g->ldu = round_ld (std::max (kept, 1));
    g->lam_h.resize (kept);
    in.get (g->lam_h.data (), (size_t) kept * 8);
    std::vector<double> lraw (kept);
    in.get (lraw.data (), (size_t) kept * 8);
    rc = g->lam_d.alloc (std::max (kept, 1));
    if (!rc) rc = g->lraw_d.alloc (std::max (kept, 1));
    if (!rc) rc = g->U.alloc ((size_t) n * g->ldu);
    if (!rc && kept > 0) {
      if (cudaMemcpy (g->lam_d.p, g->lam_h.data (), (size_t) kept * 8,
                      cudaMemcpyHostToDevice) != cudaSuccess
          || cudaMemcpy (g->lraw_d.p, lraw.data (), (size_t) kept * 8,
                         cudaMemcpyHostToDevice) != cudaSuccess
          || cudaMemset (g->U.p, 0, (size_t) n * g->ldu * 8) != cudaSuccess)
        rc = set_error (LGH_ERR_GPU, "lgh_glr_load: copy");
      if (!rc) rc = get_rows (in, g->U.p, n, kept, g->ldu);
    }
    if (!rc && ell > 0) {
      g->ell = ell;
      g->ldq = round_ld (ell);
      DBuf<double> q;
      rc = q.alloc ((size_t) n * g->ldq);
      if (!rc && cudaMemset (q.p, 0, (size_t) n * g->ldq * 8) != cudaSuccess)
        rc = set_error (LGH_ERR_GPU, "lgh_glr_load: memset");
      if (!rc) rc = get_rows (in, q.p, n, ell, g->ldq);
      std::vector<double> A ((size_t) ell * ell);
      in.get (A.data (), A.size () * 8);
      if (!rc) rc = g->A.alloc (A.size ());
      if (!rc && cudaMemcpy (g->A.p, A.data (), A.size () * 8,
                             cudaMemcpyHostToDevice) != cudaSuccess)
        rc = set_error (LGH_ERR_GPU, "lgh_glr_load: copy");
      if (!rc && prec == LGH_PREC_MIXED) {
        rc = g->Q32.alloc ((size_t) n * g->ldq);
        if (!rc) rc = launch_f64_to_f32 (n, g->ldq, q.p, g->ldq, g->Q32.p, g->ldq,
                                         stream ());
        if (!rc && cudaStreamSynchronize (stream ()) != cudaSuccess)
          rc = set_error (LGH_ERR_GPU, "lgh_glr_load: convert");
      } else if (!rc) {
        g->Q.swap (q);
      }
    }
    if (!rc && prec == LGH_PREC_MIXED && kept > 0) {
      rc = g->U32.alloc ((size_t) n * g->ldu);
      if (!rc) rc = launch_f64_to_f32 (n, g->ldu, g->U.p, g->ldu, g->U32.p, g->ldu,
                                       stream ());
    }
    const uint64_t expect = in.h;
    uint64_t sum = 0;
    if (!rc && in.ok && fread (&sum, 1, 8, in.f) != 8) in.ok = false;
    if (!rc && !in.ok)
      rc = set_error (LGH_ERR_ARG_WRONG, "lgh_glr_load: %s is truncated", path);
    if (!rc && sum != expect)
      rc = set_error (LGH_ERR_ARG_WRONG, "lgh_glr_load: checksum mismatch in %s",
                      path);
    g->stats.n = n;
    g->stats.ell = ell;
    g->stats.kept = kept;
    g->stats.precision = prec;
  }
  fclose (in.f);
  if (!rc && cudaDeviceSynchronize () != cudaSuccess)
    rc = set_error (LGH_ERR_GPU, "lgh_glr_load: device");
  if (rc) {
    if (g) lgh_glr_destroy (g);
    return rc;
  }
  *out = g;
  return 0;
}

} /* extern "C" */
