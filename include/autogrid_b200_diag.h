/*
 * autogrid_b200_diag.h -- measurement helpers of the map engine (not part of
 * the reference-facing ABI in autogrid_b200.h).
 */
#ifndef AUTOGRID_B200_DIAG_H
#define AUTOGRID_B200_DIAG_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
/* Peak issue rates of this GPU, measured with CUDA events on dependent-free
 * instruction streams: rsqrt.approx.f32 per second (the MUFU pipe the e-map
 * kernel is bound by) and FP32 FMA flops per second (2 per FMA). */
int ag_diag_peak_rates(int32_t device, double *rsqrt_per_s, double *fp32_flops_per_s, double *sm_clock_mhz);
/* Largest relative error of rsqrt.approx.f32 over every float x in
 * [2^lo_exp, 2^hi_exp), in units of 2^-24: max |rsqrt(x)*sqrt(x) - 1| / 2^-24
 * with the product and sqrt in FP64.  The far-field bin guard assumes 2.5
 * over the distances it sees ([2^20, 2^27) in squared bins). */
int ag_diag_rsqrt_error(int32_t device, int32_t lo_exp, int32_t hi_exp, double *max_rel_ulps);

/* Far-field table bins of the listed grid points (linear indices into the
 * problem's grid, X fastest) against every atom, computed with the far-field
 * kernel's own arithmetic.  Outputs [n_points][n_atoms] (host memory):
 *   bin_used  the bin the e map carries for the pair: floor(t*(1-d)) of the
 *             FP32 distance t = A_DIV*r, or the FP64-resolved bin when the
 *             guard flagged the pair; -1 for pairs nearer than 8 A (the
 *             near-field kernel's);
 *   bin_fp32  floor(t), the plain FP32 bin;
 *   flags     1: the guard flagged the pair, | 2: its FP64 squared distance
 *             lay within 1e-12 of the edge (reference expression decided).
 * At most 2^27 pairs per call.  Returns an ag_status. */
struct ag_context;
struct ag_problem;
int ag_diag_far_bins(struct ag_context *ctx, const struct ag_problem *problem, int32_t n_points,
                     const int64_t *points, int32_t *bin_used, int32_t *bin_fp32, int32_t *flags);
#ifdef __cplusplus
}
#endif
#endif
