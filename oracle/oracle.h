/* TEST INFRASTRUCTURE ONLY -- the CPU checker for the Kirchhoff summation path.
 *
 * A plain-C restatement of the reference's diffraction summation
 * (src/migration_kernel.cpp:17-383 of sergeevsn/poststackmig3d) and of the per-output-inline
 * buffer/velocity/padding rules its driver applies (src/main.cpp:188-217, 258-369;
 * src/migration_kernel.cpp:385-511).  Only tests/, the smoke check and bench.py's CPU
 * baseline may load it, and only to check or time against; the product never calls it.
 *
 * Parity of this restatement is pinned against the reference itself, compiled from its own
 * sources by oracle/Makefile into oracle/_ref/, through the committed fixtures in
 * tests/golden/ (made by tests/golden/make_golden.py).
 */
#ifndef PSM_ORACLE_H
#define PSM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* flags */
#define ORACLE_CONTRACT 1 /* evaluate r2, t2 and the weight denominator as single-rounding
                             fused multiply-adds, as GCC contracts them under
                             -ffp-contract=fast (the reference's build) */
#define ORACLE_F64 2      /* masks in the reference's FP32 arithmetic, every value (t, frac,
                             interpolation, weight, sum) in FP64: the FP64 oracle of the same
                             operator */
#define ORACLE_AVX_ORDER 4 /* FP32 sum in the reference AVX path's order (8 lane partial sums
                              per inline, remainder first, migration_kernel.cpp:188-327) */

/* kirchhoffKernel3DWithPadding restated, serial-build semantics.  Arguments mean what they
 * mean in include/migration_kernel.h:16-31; output is flat [n_out_xl][n_t].  out64 (may be
 * NULL) receives the FP64 sums when ORACLE_F64 is set.  Returns the number of accumulated
 * terms. */
int64_t oracle_kirchhoff_inline(const float *buf, int64_t n_buf_il, int64_t n_buf_xl,
                                int64_t n_t, const float *vel, float *out, double *out64,
                                int64_t n_out_xl, const int32_t *il_pos,
                                int32_t cur_il_pos, int32_t cur_xl_start, float dt,
                                const float *t0, float tan2, float d_il, float d_xl,
                                int amp, int flags);

/* The whole migration of a resident cube, as the reference driver runs it:
 *   data, vrms   [n_il][n_xl][n_t] on the real input grid
 *   out_center   [n_oi] real inline index each output inline migrates (main.cpp:258-288)
 *   out          [n_oi][n_ox][n_t]; out64 likewise in FP64 (either may be NULL)
 * Buffer inlines per output inline: [max(0,c-m_il-pad_il), min(n_il,c+m_il+1+pad_il))
 * (migration_kernel.cpp:404-409); buffer crosslines [0, n_xl+2*pad_xl) with real data at
 * [pad_xl, pad_xl+n_xl) and zeros elsewhere; padded crosslines carry v = 0.
 * counts[0] = all accumulated terms (zero padding traces included), counts[1] = terms on
 * real input traces only.  Parallel over output traces with n_threads OpenMP threads
 * (0 = default). */
void oracle_migrate_volume(const float *data, const float *vrms, int32_t n_il, int32_t n_xl,
                           int32_t n_t, const int32_t *out_center, int32_t n_oi,
                           int32_t n_ox, int32_t pad_il, int32_t pad_xl, int32_t m_il,
                           float dt, const float *t0, float tan2, float d_il, float d_xl,
                           int amp, int flags, int n_threads, float *out, double *out64,
                           int64_t *counts);

/* Real-trace term counts of output rows [r0, r1) (rows_out[r1-r0]) with the masks of
 * oracle_migrate_volume, without the summation. */
void oracle_count_rows(const float *vrms, int32_t n_il, int32_t n_xl, int32_t n_t,
                       const int32_t *out_center, int32_t r0, int32_t r1, int32_t n_ox,
                       int32_t pad_il, int32_t pad_xl, int32_t m_il, float dt,
                       const float *t0, float tan2, float d_il, float d_xl, int amp,
                       int flags, int n_threads, int64_t *rows_out);

/* Transpose of oracle_migrate_volume's linear map (FP64): data_out[n_il][n_xl][n_t]
 * receives sum over terms of (weights) * image.  Same masks as the forward. */
void oracle_adjoint_volume(const double *image, const float *vrms, int32_t n_il,
                           int32_t n_xl, int32_t n_t, const int32_t *out_center,
                           int32_t n_oi, int32_t n_ox, int32_t pad_il, int32_t pad_xl,
                           int32_t m_il, float dt, const float *t0, float tan2, float d_il,
                           float d_xl, int amp, int flags, int n_threads, double *data_out);

#ifdef __cplusplus
}
#endif
#endif
