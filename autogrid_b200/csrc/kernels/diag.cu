// Microbenchmarks for the roofline denominators: MUFU rsqrt rate and FP32 FMA rate.
#include <algorithm>
#include <cstring>
#include <cuda_runtime.h>

#include "agb_device.cuh"
#include "autogrid_b200_diag.h"

namespace agb {

__global__ void __launch_bounds__(256) k_peak_rsqrt(float *out, int iters)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = 1.0f + 1e-3f * (threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = rsqrt_approx(a[k]);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == 12345.f) out[threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_peak_ffma(float *out, int iters)
{
    float2 a[8];
    const float2 m = make_float2(0.9999f, 0.9999f), c = make_float2(1e-4f, 1e-4f);
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = make_float2(1.0f + k, 2.0f + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = __ffma2_rn(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k].x + a[k].y;
    if (s == 12345.f) out[threadIdx.x] = s;
}

// Relative error of rsqrt.approx.f32 at every float of [2^lo_exp, 2^hi_exp):
// the largest |rsqrt(x)*sqrt(x) - 1| (FP64) as order-preserving bits of a
// non-negative double.
__global__ void __launch_bounds__(256) k_rsqrt_error(uint32_t bits0, uint32_t n, unsigned long long *max_bits)
{
    double worst = 0.0;
    for (uint32_t i = blockIdx.x * 256u + threadIdx.x; i < n; i += gridDim.x * 256u) {
        const float x = __uint_as_float(bits0 + i);
        const double e = fabs((double)rsqrt_approx(x) * sqrt((double)x) - 1.0);
        worst = fmax(worst, e);
    }
    for (int o = 16; o; o >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
    if ((threadIdx.x & 31) == 0) atomicMax(max_bits, (unsigned long long)__double_as_longlong(worst));
}

}  // namespace agb

extern "C" int ag_diag_rsqrt_error(int32_t device, int32_t lo_exp, int32_t hi_exp, double *max_rel_ulps)
{
    if (!max_rel_ulps || lo_exp < -126 || hi_exp > 127 || lo_exp >= hi_exp) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 1;
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, sizeof *d) != cudaSuccess) return 1;
    cudaMemset(d, 0, sizeof *d);
    const uint32_t b0 = (uint32_t)(lo_exp + 127) << 23, b1 = (uint32_t)(hi_exp + 127) << 23;
    agb::k_rsqrt_error<<<4096, 256>>>(b0, b1 - b0, d);
    unsigned long long h = 0;
    const cudaError_t e = cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return 1;
    double v;
    std::memcpy(&v, &h, sizeof v);
    *max_rel_ulps = v * 16777216.0;
    return 0;
}

extern "C" int ag_diag_peak_rates(int32_t device, double *rsqrt_per_s, double *fp32_flops_per_s,
                                  double *sm_clock_mhz)
{
    if (cudaSetDevice(device) != cudaSuccess) return 1;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 1;
    float *out = nullptr;
    if (cudaMalloc(&out, 1024 * sizeof(float)) != cudaSuccess) return 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
    double best_r = 0, best_f = 0;
    for (int rep = 0; rep < 3; rep++) {
        float ms = 0;
        cudaEventRecord(e0);
        agb::k_peak_rsqrt<<<blocks, threads>>>(out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms > 0) best_r = std::max(best_r, (double)blocks * threads * iters * 8 / (ms * 1e-3));
        cudaEventRecord(e0);
        agb::k_peak_ffma<<<blocks, threads>>>(out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms > 0) best_f = std::max(best_f, (double)blocks * threads * iters * 8 * 2 * 2 / (ms * 1e-3));
    }
    int clk_khz = 0;
    cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (rsqrt_per_s) *rsqrt_per_s = best_r;
    if (fp32_flops_per_s) *fp32_flops_per_s = best_f;
    if (sm_clock_mhz) *sm_clock_mhz = clk_khz / 1000.0;
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
