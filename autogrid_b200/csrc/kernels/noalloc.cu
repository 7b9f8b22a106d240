// Electrostatic map with no device allocation: ag_emap_compute_noalloc().
//
// Some callers cannot call cudaMalloc: a host process that has handed the
// whole device to its own pool allocator, a real-time or serving loop where an
// allocation (and the implicit device synchronisation of cudaFree) is not
// allowed between requests, or an embedding in which only caller-owned
// buffers may be touched.  For them this file provides one entry point that
// computes the electrostatic map (LOOP 1 of the reference, main.cpp:2940-2982)
// from caller-owned device inputs into a caller-owned device output, and keeps
// its scratch (per-atom staging copies, the energy table and the per-chunk
// partial sums) in one file-scope __device__ array of fixed size.
//
// It is a variant of k_emap_far (emap.cu): the same frame decomposition,
// canonical FP32 distances, bin guard and shared-memory table gather, but it
// also covers the pairs nearer than 8 A itself -- those, and the far pairs
// the bin guard flags, are evaluated in FP64 with the reference's LOOP 1
// expression -- so it needs no near-field kernel, cell list or
// closest-hydrogen buffer.  Table bins are the reference's (pairs within
// 1e-12 of an edge in FP64 aside, where CUDA's hypot decides); this entry
// point reports no statistics.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "agb_device.cuh"

namespace agb {
void set_last_error(const std::string &m);
bool device_accessible(const void *ptr, int device);

// 32 MiB, held by every GPU that loads the library until the process exits.
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NA_THREADS = 256, NA_TILE = 512;
constexpr float NA_NEAR_T = 1026.0f;  // t = A_DIV*r below this: FP64 pair (covers the FP32 error at 8 A)

struct NoallocLayout {
    double *x128, *y128, *z128;
    float *qw, *tab, *partial;
    int chunks, chunk_atoms;
};

__global__ void k_noalloc_prep(const double *__restrict__ coord, const double *__restrict__ charge, int n_atoms,
                               int dddiel, const double *__restrict__ reps, double invdielcal, double coeff_estat,
                               NoallocLayout L)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_atoms) {
        L.x128[i] = coord[3 * i] * AG_A_DIV;
        L.y128[i] = coord[3 * i + 1] * AG_A_DIV;
        L.z128[i] = coord[3 * i + 2] * AG_A_DIV;
        L.qw[i] = (float)(charge[i] * coeff_estat * AG_A_DIV);
    }
    if (i < AG_NDIEL) L.tab[i] = (float)(dddiel ? reps[i] : invdielcal);
}

// Reference LOOP 1 term of one pair in FP64 (main.cpp:2951-2977).
__device__ __forceinline__ double loop1_term(const double *coord, const double *charge, int a, double cx, double cy,
                                             double cz, int dddiel, const double *reps, double invdielcal,
                                             double coeff_estat)
{
    double r = hypot(__dsub_rn(coord[3 * a], cx), hypot(__dsub_rn(coord[3 * a + 1], cy), __dsub_rn(coord[3 * a + 2], cz)));
    if (r < 1.0e-6) r = 1.0e-6;
    const double inv_rmax = __ddiv_rn(1.0, r > 0.5 ? r : 0.5);
    int k = (int)__dmul_rn(r, (double)AG_A_DIV);
    if (k > AG_NDIEL - 1) k = AG_NDIEL - 1;
    const double f = dddiel ? reps[k] : invdielcal;
    return __dmul_rn(__dmul_rn(__dmul_rn(charge[a], inv_rmax), f), coeff_estat);
}

__global__ void __launch_bounds__(NA_THREADS)
k_emap_noalloc(const double *__restrict__ coord, const double *__restrict__ charge, int n_atoms, int dddiel,
               const double *__restrict__ reps, double invdielcal, double coeff_estat, double spacing,
               int n1x, int n1y, int n1z, int nex, int ney, int nez, int nfx, int nfy, long long P, NoallocLayout L,
               float edge_lo, float edge_hi)
{
    extern __shared__ float4 na_smem[];
    float *s_tab = (float *)na_smem;
    float4 *s_atom = na_smem + AG_NDIEL / 4;
    const int tid = threadIdx.x;
    for (int i = tid; i < AG_NDIEL; i += NA_THREADS) s_tab[i] = L.tab[i];
    const double sp128 = spacing * AG_A_DIV;
    const int f = blockIdx.x;
    const int fx = f % nfx, fy = (f / nfx) % nfy, fz = f / (nfx * nfy);
    const int ox = fx * FRAME_X, oy = fy * FRAME_Y, oz = fz * FRAME_Z;
    const double X0 = frame_origin_bins(ox, nex, sp128), Y0 = frame_origin_bins(oy, ney, sp128),
                 Z0 = frame_origin_bins(oz, nez, sp128);
    const int lane = tid & 31, w = tid >> 5;
    const int tx = lane & 3, ty = ((lane >> 2) & 3) + 4 * (w & 1), tz = (lane >> 4) + 2 * (w >> 1);
    const float py = frame_point_coord(ty, sp128), pz = frame_point_coord(tz, sp128);
    float px[8];
    double cxp[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        px[k] = frame_point_coord(tx + 4 * k, sp128);
        cxp[k] = (double)(ox + tx + 4 * k - nex) * spacing;
    }
    const double cy = (double)(oy + ty - ney) * spacing, cz = (double)(oz + tz - nez) * spacing;
    float tot[8];
#pragma unroll
    for (int k = 0; k < 8; k++) tot[k] = 0.f;
    const int a_begin = blockIdx.y * L.chunk_atoms, a_end = min(n_atoms, a_begin + L.chunk_atoms);
    for (int a0 = a_begin; a0 < a_end; a0 += NA_TILE) {
        const int na = min(NA_TILE, a_end - a0);
        __syncthreads();
        for (int i = tid; i < NA_TILE; i += NA_THREADS) {
            float4 v = make_float4(1.0e6f, 1.0e6f, 1.0e6f, 0.f);
            if (i < na) {
                const int a = a0 + i;
                v = make_float4(frame_atom_coord(L.x128[a], X0), frame_atom_coord(L.y128[a], Y0),
                                frame_atom_coord(L.z128[a], Z0), __int_as_float(a));
            }
            s_atom[i] = v;
        }
        __syncthreads();
        float acc[8];
#pragma unroll
        for (int k = 0; k < 8; k++) acc[k] = 0.f;
        for (int i = 0; i < na; i++) {
            const float4 A = s_atom[i];
            const int a = __float_as_int(A.w);
            const float s = far_pair_s(A.y, A.z, py, pz);
            const float qa = L.qw[a];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const float dx = __fsub_rn(A.x, px[k]);
                const float t2 = __fmaf_rn(dx, dx, s);
                const float rs = rsqrt_approx(t2);
                const float t = fminf(__fmul_rn(t2, rs), FAR_CLAMP_T);
                // the far kernel's bin guard: a pair within the FP32 error bound
                // of a bin edge takes the FP64 term, with the reference's bin
                const uint32_t lo = __float_as_uint(__fmaf_rz(t, edge_lo, 8388608.f));
                const uint32_t hi = __float_as_uint(__fmaf_rz(t, edge_hi, 8388608.f));
                if (t < NA_NEAR_T || lo != hi) {
                    acc[k] += (float)loop1_term(coord, charge, a, cxp[k], cy, cz, dddiel, reps, invdielcal, coeff_estat);
                } else {
                    acc[k] = __fmaf_rn(qa * rs, s_tab[lo - MAGIC_BITS], acc[k]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) tot[k] += acc[k];
    }
    const int iy = oy + ty, iz = oz + tz;
    if (iy < n1y && iz < n1z) {
        float *out = L.partial + (size_t)blockIdx.y * (size_t)P + ((size_t)iz * n1y + iy) * (size_t)n1x;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int ix = ox + tx + 4 * k;
            if (ix < n1x) out[ix] = tot[k];
        }
    }
}

__global__ void k_noalloc_reduce(NoallocLayout L, long long P, float *__restrict__ emap)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    float e = 0.f;
    for (int c = 0; c < L.chunks; c++) e += L.partial[(size_t)c * (size_t)P + (size_t)i];
    emap[i] = e;
}

namespace {
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {};  // device address of g_noalloc_scratch, per device ordinal

// Guard multipliers of the far kernel's bin guard for this spacing (bins):
// the largest frame point coordinate and whether the frame point
// coordinates are exact floats (see far_edge_multipliers).
void noalloc_guard(double spacing_adiv, float *lo, float *hi)
{
    bool exact = true;
    for (int il = 0; il < FRAME_X; il++) {
        const double v = (double)il * spacing_adiv;
        exact &= std::fma((double)il, spacing_adiv, -v) == 0.0 && (double)(float)v == v;
    }
    const double px = (FRAME_X - 1) * spacing_adiv, pyz = (FRAME_Y - 1) * spacing_adiv;
    far_edge_multipliers(std::sqrt(px * px + 2 * pyz * pyz), exact, 2.5, lo, hi);
}

// The caller's current device, given back when the entry point returns.
struct RestoreDevice {
    int prev = -1;
    RestoreDevice() { cudaGetDevice(&prev); }
    ~RestoreDevice()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};
}

}  // namespace agb

extern "C" ag_status ag_emap_compute_noalloc(int32_t device, int32_t n_atoms, const double *d_coord,
                                             const double *d_charge, const int32_t n1[3], double spacing,
                                             int32_t dddiel, const double *d_r_epsilon_fn, double invdielcal,
                                             double coeff_estat, float *d_emap, void *stream)
{
    using namespace agb;
    if (!n1 || !d_emap || (n_atoms > 0 && (!d_coord || !d_charge)) || (dddiel && !d_r_epsilon_fn)) {
        set_last_error("ag_emap_compute_noalloc: null argument");
        return AG_ERR_INVALID;
    }
    if (device < 0 || device >= 64) {
        set_last_error("ag_emap_compute_noalloc: device ordinal out of range");
        return AG_ERR_INVALID;
    }
    for (int i = 0; i < 3; i++)
        if (n1[i] < 1 || n1[i] > AG_MAX_GRID_PTS + 1 || n1[i] % 2 != 1) {
            set_last_error("ag_emap_compute_noalloc: n1 must be odd and within [1, MAX_GRID_PTS+1]");
            return AG_ERR_INVALID;
        }
    if (n_atoms < 0 || n_atoms > AG_MAX_ATOMS) {
        set_last_error("ag_emap_compute_noalloc: n_atoms out of range [0, AG_MAX_ATOMS]");
        return AG_ERR_TOO_LARGE;
    }
    if (!(spacing > 0.0)) {
        set_last_error("ag_emap_compute_noalloc: spacing must be positive");
        return AG_ERR_INVALID;
    }
    const long long P = (long long)n1[0] * n1[1] * n1[2];
    // scratch carve-up, each piece 256-byte aligned
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t atoms_bytes = up(sizeof(double) * (size_t)std::max(n_atoms, 1)) * 3 + up(sizeof(float) * (size_t)std::max(n_atoms, 1));
    const size_t tab_bytes = up(sizeof(float) * AG_NDIEL);
    const size_t fixed = atoms_bytes + tab_bytes;
    if (fixed + up(sizeof(float) * (size_t)P) > NOALLOC_SCRATCH_BYTES) {
        set_last_error("ag_emap_compute_noalloc: grid of " + std::to_string(P) + " points with " +
                       std::to_string(n_atoms) + " atoms exceeds the 32 MiB no-allocation scratch (about " +
                       std::to_string((NOALLOC_SCRATCH_BYTES - fixed) / sizeof(float)) + " points)");
        return AG_ERR_TOO_LARGE;
    }
    if (!device_accessible(d_emap, device) || (n_atoms > 0 && (!device_accessible(d_coord, device) ||
                                                              !device_accessible(d_charge, device))) ||
        (dddiel && !device_accessible(d_r_epsilon_fn, device))) {
        set_last_error("ag_emap_compute_noalloc: the buffers must be device memory of the given GPU");
        return AG_ERR_INVALID;
    }
    RestoreDevice restore;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        set_last_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        return AG_ERR_CUDA;
    }
    if (stream) {
        int sdev = -1;
        e = cudaStreamGetDevice((cudaStream_t)stream, &sdev);
        if (e != cudaSuccess || sdev != device) {
            set_last_error("ag_emap_compute_noalloc: the stream does not belong to the given device");
            return AG_ERR_INVALID;
        }
    }
    void *base = nullptr;
    {
        // once per device, with that device current: the host-side symbol is a
        // stand-in, only cudaGetSymbolAddress yields the device address
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[device]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return AG_ERR_CUDA;
            }
            g_noalloc_ptr[device] = p;
        }
        base = g_noalloc_ptr[device];
    }
    NoallocLayout L;
    unsigned char *b = (unsigned char *)base;
    const size_t na = (size_t)std::max(n_atoms, 1);
    L.x128 = (double *)b; b += up(sizeof(double) * na);
    L.y128 = (double *)b; b += up(sizeof(double) * na);
    L.z128 = (double *)b; b += up(sizeof(double) * na);
    L.qw = (float *)b; b += up(sizeof(float) * na);
    L.tab = (float *)b; b += tab_bytes;
    L.partial = (float *)b;
    const int nfx = (n1[0] + FRAME_X - 1) / FRAME_X, nfy = (n1[1] + FRAME_Y - 1) / FRAME_Y, nfz = (n1[2] + FRAME_Z - 1) / FRAME_Z;
    const long long frames = (long long)nfx * nfy * nfz;
    const size_t max_chunks = (NOALLOC_SCRATCH_BYTES - fixed) / up(sizeof(float) * (size_t)P);
    int chunks = (int)std::max(1LL, ((long long)current_device_sms() * 8 * 3 + frames - 1) / frames);
    chunks = (int)std::min<long long>(chunks, (long long)max_chunks);
    chunks = std::min(chunks, std::max(1, (n_atoms + NA_TILE - 1) / NA_TILE));
    L.chunk_atoms = ((std::max(n_atoms, 1) + chunks - 1) / chunks + NA_TILE - 1) / NA_TILE * NA_TILE;
    L.chunks = std::max(1, (n_atoms + L.chunk_atoms - 1) / L.chunk_atoms);
    cudaStream_t s = (cudaStream_t)stream;
    const int prep_n = std::max(n_atoms, AG_NDIEL);
    k_noalloc_prep<<<(prep_n + 255) / 256, 256, 0, s>>>(d_coord, d_charge, n_atoms, dddiel, d_r_epsilon_fn, invdielcal,
                                                       coeff_estat, L);
    if (n_atoms > 0) {
        const size_t smem = AG_NDIEL * sizeof(float) + NA_TILE * sizeof(float4);
        e = cudaFuncSetAttribute(k_emap_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        float edge_lo = 1.f, edge_hi = 1.f;
        noalloc_guard(spacing * AG_A_DIV, &edge_lo, &edge_hi);
        if (e == cudaSuccess) {
            k_emap_noalloc<<<dim3((unsigned)frames, (unsigned)L.chunks), NA_THREADS, smem, s>>>(
                d_coord, d_charge, n_atoms, dddiel, d_r_epsilon_fn, invdielcal, coeff_estat, spacing, n1[0], n1[1],
                n1[2], (n1[0] - 1) / 2, (n1[1] - 1) / 2, (n1[2] - 1) / 2, nfx, nfy, P, L, edge_lo, edge_hi);
        }
    } else {
        L.chunks = 0;  // no atoms: the map is zero
    }
    if (e == cudaSuccess) {
        k_noalloc_reduce<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(L, P, d_emap);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("ag_emap_compute_noalloc launch: ") + cudaGetErrorString(e));
        return AG_ERR_CUDA;
    }
    return AG_OK;
}
