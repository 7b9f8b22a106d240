// Launchers of the map-text kernels (kernels/maptext.cu).
#pragma once
#include <cuda_runtime.h>

namespace agb {

struct TextArgs {
    const float *m32;    // one of m32 / m64: n_out maps of P values
    const double *m64;
    long long P;
    int n_out;           // maps formatted
    int n_energy;        // maps [0, n_energy) are energy maps
    int floating;        // 1: map n_energy is the floating grid; the rest are counts
    int bpm;             // blocks per map (text_blocks_per_map(P))
    unsigned char *len8;            // [n_out*bpm*text_values_per_block()] line lengths
    unsigned *blk_len;              // [n_out*bpm] bytes per block
    unsigned long long *blk_off;    // [n_out*bpm] text offset of each block
    unsigned long long *ext;        // [2*n_energy] order keys of min, max
    unsigned long long *map_bytes;  // [n_out+1] bytes per map, then the total
    char *text;                     // [total] output
};

int text_blocks_per_map(long long P);
long long text_values_per_block();
// k_text_init + k_text_measure + k_text_scan (fills len8, blk_len, blk_off, ext, map_bytes)
cudaError_t launch_text_measure(const TextArgs &a, cudaStream_t s);
// k_text_write (needs the measure launches and a.text of map_bytes[n_out] bytes)
cudaError_t launch_text_write(const TextArgs &a, cudaStream_t s);

// host decoding of the extrema keys
inline double text_key_to_double(unsigned long long k)
{
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double d;
    __builtin_memcpy(&d, &b, 8);
    return d;
}

}  // namespace agb
