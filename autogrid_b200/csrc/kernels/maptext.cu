// Map-file bodies on the device: the text loop of main.cpp:3481-3519, one
// line per grid point of each output map, formatted by kernels/maptext.cuh.
//
// Three launches:
//   k_text_measure  line lengths (one byte per value), bytes per block of
//                   TXT_VPB values, and the extrema of each energy map
//                   (main.cpp:3494-3495) as order-preserving 64-bit keys;
//   k_text_scan     one CTA: exclusive prefix sum of the block byte counts,
//                   bytes per map and in total;
//   k_text_write    each block formats its values into shared memory at the
//                   offsets of a block scan of the lengths, then copies its
//                   bytes to the text buffer with coalesced stores.
// A block never spans two maps, so each map's body is contiguous and ends
// where the next begins.
#include <cuda_runtime.h>

#include "kernels/maptext.cuh"
#include "kernels/maptext.h"

namespace agb {

namespace {

constexpr int TXT_THREADS = 256;
constexpr int TXT_VPT = 2;
constexpr int TXT_VPB = TXT_THREADS * TXT_VPT;
constexpr int SCAN_THREADS = 1024;

__device__ __forceinline__ unsigned long long order_key(double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double value_at(const TextArgs &a, int map, long long i)
{
    const long long k = (long long)map * a.P + i;
    return a.m64 ? a.m64[k] : (double)a.m32[k];
}

__device__ __forceinline__ int line_kind(const TextArgs &a, int map)
{
    if (map < a.n_energy) return agt::kEnergy;
    if (a.floating && map == a.n_energy) return agt::kFloating;
    return agt::kCount;
}

// Inclusive warp scan, then block exclusive scan; returns this thread's
// exclusive prefix and the block total through *total.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned *warp_sums, unsigned *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned s = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) warp_sums[lane] = s;  // inclusive
    }
    __syncthreads();
    const unsigned before = (w ? warp_sums[w - 1] : 0u) + x - v;
    *total = warp_sums[nw - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(TXT_THREADS) k_text_init(TextArgs a)
{
    for (int i = threadIdx.x; i < a.n_energy; i += blockDim.x) {
        a.ext[2 * i] = order_key(__longlong_as_double(0x7ff0000000000000ll));       // min <- +inf
        a.ext[2 * i + 1] = order_key(__longlong_as_double((long long)0xfff0000000000000ull));  // max <- -inf
    }
}

__global__ void __launch_bounds__(TXT_THREADS) k_text_measure(TextArgs a)
{
    __shared__ unsigned warp_sums[TXT_THREADS / 32];
    __shared__ double wmin[TXT_THREADS / 32], wmax[TXT_THREADS / 32];
    const int b = blockIdx.x;
    const int map = b / a.bpm;
    const long long base = (long long)(b - map * a.bpm) * TXT_VPB;
    const int kind = line_kind(a, map);
    unsigned len = 0;
    double lo = __longlong_as_double(0x7ff0000000000000ll), hi = -lo;
#pragma unroll
    for (int i = 0; i < TXT_VPT; i++) {
        const long long idx = base + threadIdx.x + (long long)i * TXT_THREADS;
        if (idx < a.P) {
            const double e = value_at(a, map, idx);
            const int n = agt::format_line(kind, e, nullptr);
            a.len8[(long long)b * TXT_VPB + threadIdx.x + i * TXT_THREADS] = (unsigned char)n;
            len += (unsigned)n;
            lo = fmin(lo, e);
            hi = fmax(hi, e);
        }
    }
    unsigned total;
    block_exclusive_scan(len, warp_sums, &total);
    if (threadIdx.x == 0) a.blk_len[b] = total;
    if (kind == agt::kEnergy) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) {
            wmin[w] = lo;
            wmax[w] = hi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 1; k < TXT_THREADS / 32; k++) {
                lo = fmin(lo, wmin[k]);
                hi = fmax(hi, wmax[k]);
            }
            atomicMin(a.ext + 2 * map, order_key(lo));
            atomicMax(a.ext + 2 * map + 1, order_key(hi));
        }
    }
}

// One CTA.  Thread t owns blocks [t*seg, (t+1)*seg).
__global__ void __launch_bounds__(SCAN_THREADS) k_text_scan(TextArgs a, long long nb)
{
    __shared__ unsigned long long part[SCAN_THREADS];
    const long long seg = (nb + SCAN_THREADS - 1) / SCAN_THREADS;
    const long long b0 = min(nb, (long long)threadIdx.x * seg), b1 = min(nb, b0 + seg);
    unsigned long long s = 0;
    for (long long b = b0; b < b1; b++) s += a.blk_len[b];
    part[threadIdx.x] = s;
    __syncthreads();
    // Hillis-Steele inclusive scan over the per-thread sums (64-bit)
    for (int o = 1; o < SCAN_THREADS; o <<= 1) {
        const unsigned long long y = threadIdx.x >= o ? part[threadIdx.x - o] : 0ull;
        __syncthreads();
        part[threadIdx.x] += y;
        __syncthreads();
    }
    unsigned long long run = part[threadIdx.x] - s;
    for (long long b = b0; b < b1; b++) {
        a.blk_off[b] = run;
        run += a.blk_len[b];
    }
    __syncthreads();
    const unsigned long long grand = part[SCAN_THREADS - 1];
    for (int m = threadIdx.x; m < a.n_out; m += SCAN_THREADS) {
        const unsigned long long o0 = a.blk_off[(long long)m * a.bpm];
        const unsigned long long o1 = (m + 1 < a.n_out) ? a.blk_off[(long long)(m + 1) * a.bpm] : grand;
        a.map_bytes[m] = o1 - o0;
    }
    if (threadIdx.x == 0) a.map_bytes[a.n_out] = grand;
}

__global__ void __launch_bounds__(TXT_THREADS) k_text_write(TextArgs a)
{
    __shared__ unsigned warp_sums[TXT_THREADS / 32];
    __shared__ unsigned off[TXT_VPB];
    __shared__ char stage[TXT_VPB * agt::kMaxLine];
    const int b = blockIdx.x;
    const int map = b / a.bpm;
    const long long base = (long long)(b - map * a.bpm) * TXT_VPB;
    const int kind = line_kind(a, map);
    // lengths of this thread's consecutive values TXT_VPT*t .. TXT_VPT*t+TXT_VPT-1
    unsigned n[TXT_VPT], mine = 0;
#pragma unroll
    for (int i = 0; i < TXT_VPT; i++) {
        const int v = threadIdx.x * TXT_VPT + i;
        n[i] = (base + v < a.P) ? a.len8[(long long)b * TXT_VPB + v] : 0u;
        mine += n[i];
    }
    unsigned total;
    unsigned o = block_exclusive_scan(mine, warp_sums, &total);
#pragma unroll
    for (int i = 0; i < TXT_VPT; i++) {
        off[threadIdx.x * TXT_VPT + i] = o;
        o += n[i];
    }
    __syncthreads();
    // format value v (coalesced reads: v = t + i*TXT_THREADS) at its offset
#pragma unroll
    for (int i = 0; i < TXT_VPT; i++) {
        const int v = threadIdx.x + i * TXT_THREADS;
        if (base + v < a.P) agt::format_line(kind, value_at(a, map, base + v), stage + off[v]);
    }
    __syncthreads();
    char *dst = a.text + a.blk_off[b];
    for (unsigned k = threadIdx.x; k < total; k += TXT_THREADS) dst[k] = stage[k];
}

}  // namespace

int text_blocks_per_map(long long P) { return (int)((P + TXT_VPB - 1) / TXT_VPB); }
long long text_values_per_block() { return TXT_VPB; }

cudaError_t launch_text_measure(const TextArgs &a, cudaStream_t s)
{
    const long long nb = (long long)a.n_out * a.bpm;
    if (nb <= 0 || nb > 0x7fffffffll) return cudaErrorInvalidValue;
    k_text_init<<<1, TXT_THREADS, 0, s>>>(a);
    k_text_measure<<<(unsigned)nb, TXT_THREADS, 0, s>>>(a);
    k_text_scan<<<1, SCAN_THREADS, 0, s>>>(a, nb);
    return cudaGetLastError();
}

cudaError_t launch_text_write(const TextArgs &a, cudaStream_t s)
{
    const long long nb = (long long)a.n_out * a.bpm;
    if (nb <= 0 || nb > 0x7fffffffll) return cudaErrorInvalidValue;
    k_text_write<<<(unsigned)nb, TXT_THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace agb
