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
/* mixed-precision objects: the tensor-core operands and tensor maps */
int shift_plan_prepare_umma (ShiftPlan *P, lgh_glr *g, int nshift, int m);
/* the error flag of the tensor-core kernel (nonzero: a wait ran out) */
int shift_plan_check (ShiftPlan *P);
/* whether this device runs the tensor-core form (sm_100, tensor maps) */
bool umma_supported ();

/* tile variants of the combination kernel: FP64 objects 0 = 64 x 64 (4
 * warps), 1 = 128 x 64 (8 warps) on the FP64 mma.sync path; mixed objects
 * on tcgen05 (TF32 x 3): 2 = 128 x 128 and 3 = 128 x 256 with a two-stage
 * load pipeline (one CTA per SM), 4 = 128 x 128 and 5 = 128 x 256 with one
 * stage (three and two CTAs per SM, whose loads, MMAs and epilogues
 * overlap one another) */
constexpr int kShiftVariants = 2;
constexpr int kUmmaVariants = 4;
/* tcgen05 variant u = variant - kShiftVariants: tile width and stages */
inline int umma_variant_tn (int u) { return (u & 1) ? 256 : 128; }
inline int umma_variant_stages (int u) { return u >= 2 ? 1 : 2; }
int launch_shift_combine_variant (int variant, int64_t n, int kept, int m,
                                  int nshift, const double *W, int ldw,
                                  const double *C, const double *g,
                                  const double *fc, const double *Y0,
                                  int ldy0, double *const *out,
                                  const int64_t *ldo, cudaStream_t s);

/* the tensor-core (tcgen05) form of the combination for mixed-precision
 * objects (k_umma.cu): TF32 operands split in two parts, four TMA tensor
 * maps (A hi / lo: n x kpad, B hi / lo: columns x kpad, FP32, K-major) */
struct UmmaMaps
{
  alignas (64) unsigned char raw[4 * 128];
  int tn = 0;
};
int umma_split_rows (int64_t n, int kept, int kpad, const double *W, int ldw,
                     float *Ah, float *Al, cudaStream_t s);
int umma_split_coef (int kept, int kpad, int m, int nshift, int ncolp,
                     const double *g, const double *C, float *Bh, float *Bl,
                     cudaStream_t s);
int umma_encode (UmmaMaps *M, const float *Ah, const float *Al, int64_t n,
                 const float *Bh, const float *Bl, int ncolp, int kpad, int tn);
int launch_shift_combine_umma (const UmmaMaps &M, int stages, int64_t n,
                               int kpad, int m,
                               int nshift, const double *fc, const double *Y0,
                               int ldy0, double *const *out, const int64_t *ldo,
                               int *err, cudaStream_t s);

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
