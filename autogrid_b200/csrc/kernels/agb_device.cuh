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
#include <cstdint>
#include <cuda_runtime.h>

#include "autogrid_b200.h"

namespace agb {

constexpr int FRAME_X = 32, FRAME_Y = 8, FRAME_Z = 8;
constexpr int FAR_BIN0 = AG_NEINT;          // bins below this belong to the near kernel
constexpr float FAR_T0 = (float)AG_NEINT;   // t = A_DIV * r threshold, same meaning
constexpr float TINY_T2 = 1.0e-20f;         // keeps rsqrt finite for coincident points
constexpr float FAR_MAX_T = (float)(AG_NDIEL - 1);

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
};
enum { FAR_TAB_TABLE = 0, FAR_TAB_CONST = 2 };

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
