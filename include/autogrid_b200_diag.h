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
#ifdef __cplusplus
}
#endif
#endif
