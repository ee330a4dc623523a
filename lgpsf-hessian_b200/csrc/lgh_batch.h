/* lgh_batch.h -- the many-shift combination stage (batch.cu) and the
 * autotuner that picks its tile shape (tune.cu). */

#ifndef LGH_BATCH_H
#define LGH_BATCH_H

#include "lgh_internal.h"

struct lgh_glr;

namespace lgh
{

struct ShiftPlan;

/* the object's plan, its workspace sized for n rows, m columns, kept
 * modes and nshift shifts */
int shift_plan_get (lgh_glr *g, int64_t n, int m, int kept, int nshift,
                    ShiftPlan **out);
double *shift_plan_R (ShiftPlan *P);
double *shift_plan_Xs (ShiftPlan *P);
double *shift_plan_Y0 (ShiftPlan *P);
double *shift_plan_Wc (ShiftPlan *P);
double *shift_plan_work (ShiftPlan *P, size_t *elems);
/* x (column-major, nshift blocks of m columns, leading dimension ldx) from
 * the plan's Y0 and Wc and the object's W; kind 0 solve, 1 sample */
int shift_plan_combine (ShiftPlan *P, lgh_glr *g, int kind, int nshift,
                        const double *c_host, int m, double *x, int64_t ldx,
                        int variant);
int shift_plan_run_eager (ShiftPlan *P, lgh_glr *g, int kind, int nshift,
                          const double *c_host, int m, double *x, int64_t ldx,
                          int variant);
void shift_plan_stats (const ShiftPlan *P, long *captures, long *replays,
                       int *last_variant);
void shift_plan_free (ShiftPlan *P);

/* tile variants of the combination kernel: 0 = 64 x 64 (4 warps),
 * 1 = 128 x 64 (8 warps) */
constexpr int kShiftVariants = 2;
int launch_shift_combine_variant (int variant, int64_t n, int kept, int m,
                                  int nshift, const double *W, int ldw,
                                  const double *C, const double *g,
                                  const double *fc, const double *Y0,
                                  int ldy0, double *const *out,
                                  const int64_t *ldo, cudaStream_t s);

/* the autotuner: the fastest variant for a shape key, measured once per
 * process (and kept in the cache file named by LGH_TUNE_CACHE, when set);
 * `trial(v)` runs variant v once on the caller's stream */
typedef int (*tune_trial_fn) (int variant, void *ctx);
int tune_pick (const char *op, int64_t n, int kept, int m, int nshift,
               int nvariants, tune_trial_fn trial, void *ctx, int *variant,
               int *measured);
/* entries of the tuner's table (for tests and reports) */
int tune_table_size ();

} /* namespace lgh */

#endif /* LGH_BATCH_H */
