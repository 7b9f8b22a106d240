// Device-side data layout and shared arithmetic of the map kernels.
//
// Frames.  The grid is tiled into frames of FRAME_X x FRAME_Y x FRAME_Z points.
// Inside a frame, atom and grid-point coordinates are expressed relative to
// the frame's first point, in units of distance-table bins (1/A_DIV Angstrom),
// and rounded to FP32 by one canonical routine.  The far-field e-map kernel
// and the near-field (short-range) kernel both decide "is this pair far?"
// from exactly the same FP32 operations on exactly the same FP32 inputs, so
// every (point, atom) pair is counted by exactly one of them.
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "autogrid_b200.h"

namespace agb {

constexpr int FRAME_X = 32, FRAME_Y = 8, FRAME_Z = 8;
constexpr int FAR_BIN0 = AG_NEINT;          // bins below this belong to the near kernel
constexpr float FAR_T0 = (float)AG_NEINT;   // t = A_DIV * r threshold, same meaning
constexpr float TINY_T2 = 1.0e-20f;         // keeps rsqrt finite for coincident points
constexpr float FAR_MAX_T = (float)(AG_NDIEL - 1);
// The guarded far kernel clamps t half a bin past the last table bin, so that
// both guard bins of a clamped pair are the last bin (the reference clamps
// the bin, min(lookup(r), NDIEL-1), main.cpp:2956).
constexpr float FAR_CLAMP_T = (float)(AG_NDIEL - 1) + 0.5f;
constexpr uint32_t MAGIC_BITS = 0x4B000000u;  // bits of 2^23: bits(2^23 + k) = MAGIC_BITS + k, 0 <= k < 2^23

// Frame origin in bins: ((o - ne) * spacing) * A_DIV, formed like the
// reference forms a grid coordinate (main.cpp:2859); the scaling by A_DIV = 2^7
// is exact, so this equals ((o - ne) * (spacing * A_DIV)).
__host__ __device__ inline double frame_origin_bins(int o, int ne, double spacing_adiv)
{
    return (double)(o - ne) * spacing_adiv;
}
// Canonical FP32 frame-relative coordinate of an atom from x*A_DIV (exact in
// FP64) and the frame origin in bins.
__device__ __forceinline__ float frame_atom_coord(double x_adiv, double origin_bins)
{
    return __double2float_rn(__dsub_rn(x_adiv, origin_bins));
}
// Canonical FP32 frame-relative coordinate of grid point il (local index).
__host__ __device__ inline float frame_point_coord(int il, double spacing_adiv)
{
#ifdef __CUDA_ARCH__
    return __double2float_rn(__dmul_rn((double)il, spacing_adiv));
#else
    return (float)((double)il * spacing_adiv);
#endif
}

__device__ __forceinline__ float rsqrt_approx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Square root of x >= 0 by the hardware approximation (one MUFU operation,
// a few ulp; sqrt(0) = 0).  Used for the directional factors of H-bond
// pairs, which are continuous where it is used.
__device__ __forceinline__ float sqrt_approx(float x)
{
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The far kernel's distance (in bins) of a pair, from frame-relative FP32
// inputs.  Written with explicit round-to-nearest intrinsics so no contraction
// or reassociation can make two call sites differ.
__device__ __forceinline__ float far_pair_s(float ay, float az, float py, float pz)
{
    const float dy = __fsub_rn(ay, py), dz = __fsub_rn(az, pz);
    return __fmaf_rn(dy, dy, __fmaf_rn(dz, dz, TINY_T2));
}
__device__ __forceinline__ float far_pair_t(float ax, float px, float s)
{
    const float dx = __fsub_rn(ax, px);
    const float t2 = __fmaf_rn(dx, dx, s);
    return __fmul_rn(t2, rsqrt_approx(t2));
}

// Far-field e-map kernel arguments for one instance.
struct FarArgs {
    const double *ax128, *ay128, *az128;  // x*A_DIV (exact in FP64)
    const float *qw;                      // q*coeff_estat*A_DIV
    const float *far_tab;                 // [NDIEL], zero below FAR_BIN0
    float *partial;                       // [chunks][P]
    double spacing_adiv;
    long long P;
    int n_atoms, chunk_atoms;
    int n1x, n1y, n1z, nex, ney, nez, nfx, nfy, nfz;
    int frame0;                           // single-instance launches: first frame of the launch
    // How a pair's table value T[b] (b = floor(t) >= AG_NEINT) is obtained:
    //   FAR_TAB_TABLE  shared-memory gather from far_tab, every pair;
    //   FAR_TAB_CONST  far_tab is one constant (constant dielectric): no gather.
    int tab_mode;
    float tab_const;
    // Bin-edge guard (FAR_TAB_TABLE): the kernel takes the bins of t*edge_lo
    // and t*edge_hi, edge_lo/hi = 1 -/+ d with d above the relative error of
    // the FP32 distance t, and sets a bit per (thread, atom) with a pair whose
    // two bins differ in edge_bits (edge_words 32-bit words per thread and
    // unit); the fix-up kernel gives those pairs their bin in FP64
    // (far_exact_bin).  tab_full [NDIEL]: the table without the zeros below
    // FAR_BIN0, for pairs whose exact bin is there.
    float edge_lo, edge_hi;
    const float *tab_full;
    uint32_t *edge_bits;
    int edge_words;
    // The shared-memory table: tab_len floats of far_tab (a multiple of 4).
    // clamp = 1: tab_len = NDIEL and t is clamped at FAR_CLAMP_T; clamp = 0:
    // the table repeats bin NDIEL-1 up to a length that covers every distance
    // of the instance (far_table_len), and t is used unclamped.
    int tab_len, clamp;
    // [0] guarded pairs resolved in FP64, [1] of those, pairs whose plain FP32
    // bin floor(t) was not the exact bin, [2] pairs decided by the reference's
    // own expression because their FP64 squared distance lies within 1e-12 of
    // the edge.  May be null (not counted).
    unsigned long long *edge_counters;
};
enum { FAR_TAB_TABLE = 0, FAR_TAB_CONST = 2 };
// Longest extended far table (bins): 128 A.  Instances with longer distances clamp.
constexpr int FAR_TAB_MAX = 16384;

// Guard multipliers for a grid: the relative error bound of the canonical
// FP32 distance t of a far pair (t >= FAR_T0 bins), rounded up so that 1 - d
// and 1 + d are floats.  With D the exact frame-relative distance (bins), A
// the atom's and P the point's frame-relative coordinates (|A| <= |D| + |P|):
//   coordinates rounded to FP32 and dx = A - P rounded:
//       |error vector| <= 2^-24 (|A| + |D| + |P| [P inexact]) <= 2^-24 (2|D| + (1 + [P inexact])|P|)
//   t2 = dx^2 + (dy^2 + dz^2) by two FMAs: relative 3 * 2^-24, 1.5 * 2^-24 on t
//   rsqrt.approx: relative rho;  t = t2 * rs rounded: 2^-24
// so |t/D - 1| <= 2^-24 (4.5 + (1 + [P inexact]) |P|max / FAR_T0) + rho.
// rho_ulps is rho in units of 2^-24; p_max the largest |P| of a frame point;
// p_exact whether every frame point coordinate is an exact float.
__host__ inline void far_edge_multipliers(double p_max, bool p_exact, double rho_ulps, float *lo, float *hi)
{
    const double u = 1.0 / 16777216.0;  // 2^-24
    const double d = u * (4.5 + rho_ulps + (p_exact ? 1.0 : 2.0) * p_max / (double)FAR_T0) * 1.0625;
    const double kl = std::ceil(d / u), kh = std::ceil(d / (2 * u));
    *lo = (float)(1.0 - kl * u);        // floats below 1 are spaced 2^-24
    *hi = (float)(1.0 + kh * 2 * u);    // floats above 1 are spaced 2^-23
}

// Streaming multiprocessors of the current device (launch sizing).
int current_device_sms();

// Device image of one problem instance.
struct DevProblem {
    int n_atoms, n_maps, n_atom_maps, n_rec_types;
    int elec_map, dsolv_map;
    int n1x, n1y, n1z, nex, ney, nez;
    long long P;
    double spacing;
    int dddiel, disorder_h, hydrogen_type, sep_desolv;
    double invdielcal, coeff_estat, solpar_q;
    double cov_pos[3], cov_half_width, cov_barrier;
    int any_covalent;
    int report_collisions;             // 'map_receptor_interior off' (ag_problem)

    // atoms in file order (FP64, centred)
    const double *x, *y, *z, *q, *vol, *solpar;
    const double *rv, *rv2;            // [3N]
    const int *type, *hbond, *rexp;
    const uint8_t *disorder;
    // DS/D1 atoms in file order
    int n_h;
    const int *h_index;                // [n_h] file index
    // cell list over the near region
    int ncx, ncy, ncz;
    double cell0[3], cell_size;        // origin (centred frame), edge
    const int *cell_start;             // [ncx*ncy*ncz + 1]
    const int *cell_atoms;             // [n_near] file indices sorted by cell
    // per-map constants
    const int *m_cov, *m_hb, *m_hbond;
    const double *m_solpar, *m_vol;
    // tables
    const float *vdw;                  // [types][atom_maps][NEINT]
    const double *sol_fn, *reps;       // [NDIEL]
    const float *far_tab;              // [NDIEL] 0 below FAR_BIN0, energy factor above
};

}  // namespace agb
