/* lgh_strip.h -- the strip form of a sparse operator (k_strip.cu). */

#ifndef LGH_STRIP_H
#define LGH_STRIP_H

#include "lgh_internal.h"

namespace lgh
{

/* R consecutive rows per strip; per strip the union of the rows' columns,
 * each union entry carrying R values (zero where a row has no entry) */
struct StripForm
{
  int R = 0;
  int64_t n = 0, nstrips = 0, nent = 0, nnz = 0;
  int64_t *sptr = nullptr;  /* nstrips + 1 */
  int32_t *scol = nullptr;  /* nent */
  double *sval = nullptr;   /* nent * R */
  float *sval32 = nullptr;  /* nent * R */
};

/* build from a device CSR; force_R in {2, 4, 8} or 0 (chosen by the cost
 * model from the union lengths) */
int strip_build (const Csr &A, int force_R, StripForm &S);
void strip_free (StripForm &S);

/* Y = A X on 16-byte aligned row-major blocks of width w */
template <typename T>
int launch_strip_spmm (const StripForm &S, const T *X, int ldx, T *Y, int ldy,
                       int w, cudaStream_t s);

} /* namespace lgh */

#endif /* LGH_STRIP_H */
