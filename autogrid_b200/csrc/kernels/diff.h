// Differentiable mode: the AutoGrid 4 maps of main.cpp:2805-3464 with every
// distance table read by linear interpolation between bins, plus the adjoint
// that maps dL/d(maps) to dL/d(receptor coordinates, charges, bond vectors).
//
// Definition of the mode (what the forward computes), pair (p, a) with
// d = x_a - x_p, r = |d|, x = A_DIV * r:
//   * tables: T(x) = T[b] + (x - b)(T[b+1] - T[b]), b = floor(x); past the last
//     entry a table is constant (the short-range tables stop at bin NEINT-1,
//     the dielectric table at NDIEL-1);
//   * the e map sums every atom (LOOP 1), F(r) = T_eps(x) / max(r, 0.5);
//   * short-range terms (LOOP 2, r <= 8 A) are multiplied by the switch
//     w = min(1, NEINT - x), which is 1 except over the last bin and brings
//     every term (desolvation included) to zero at the 8 A cutoff;
//   * the D1 ramp Hramp is evaluated for every D1 pair (the reference leaves it
//     at 1 when cos_theta <= 0, a jump when rsph > 0), and the A2 branch for
//     cos_theta < 0 is scaled by (1 + sin(2 ti) / 9) so both branches meet at
//     cos_theta = 0 (the reference jumps by 0.1 sin(2 ti) there);
//   * discrete choices are frozen: the closest DS/D1 hydrogen of each point can
//     be kept from an earlier evaluation, the bonded neighbours that define the
//     bond vectors are the ones found at load time, and the H-bond min/max
//     terms pass their gradient to the atom that attains them.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "autogrid_b200.h"

namespace agb {

constexpr int DF_MAXS = 16;   // map slots of the short-range kernels (atom maps, desolvation partners, d)
constexpr int DF_MAXMM = 8;   // slots that keep an H-bond min/max
constexpr int DF_LEAN_S = 8;  // slots of the lean kernel instantiations
constexpr int DF_MID_MM = 2;  // min/max registers of the middle one (the lean one has none)
constexpr int DF_BRICK_X = 8, DF_BRICK_Y = 8, DF_BRICK_Z = 4;
constexpr int DF_THREADS = DF_BRICK_X * DF_BRICK_Y * DF_BRICK_Z;
constexpr int DF_STAGE = 256;       // candidate atoms staged in shared memory at once
constexpr double DF_RADIUS = 8.05;  // cell acceptance radius (A), > the 8 A cutoff

// What a (slot, receptor class) pair adds, after main.cpp:3290-3379.
enum : uint8_t {
    DA_NONE = 0,
    DA_PLAIN,     // v = T
    DA_SUMA,      // acceptor probe, donor receptor: v = T H (racc + (1-racc) rsph)
    DA_SUMA_DIS,  // same, disordered receptor: T_H(r - 1.1) in place of T
    DA_MMA,       // NA-type probe, donor receptor: min/max of T (racc + (1-racc) rsph)
    DA_SUMD_DIS,  // donor probe, disordered acceptor: v = T_H H (rdon + (1-rdon) rsph)
    DA_MMD,       // donor probe, acceptor receptor: min/max of T (rdon + (1-rdon) rsph)
};

enum : int { DK_ATOM = 0, DK_D = 1, DK_COV = 2 };

// Conformers.  n_conf coordinate sets of one receptor (same atoms, types,
// tables and grid) are evaluated by one launch: per conformer k the arrays
// marked [conf] below start at k times their per-conformer length (x, y, z, q:
// N; rv, rv2: 3N; cell_start: ncells + 1; cell_atoms: N; maps: n_maps * P;
// closest H: P; min/max atoms: 2 * n_mm * P; gradients: 10 N).
struct DiffArgs {
    int n_atoms, n1x, n1y, n1z, nex, ney, nez;
    long long P;
    double spacing;
    int n_conf;
    // atoms in file order, centred frame, FP64
    const double *x, *y, *z, *q, *rv, *rv2;  // [conf]; rv, rv2: [3N]
    const double *vol, *solpar;
    const int *meta;          // type | hbond << 5 | rexp << 8 | disorder << 11 | skip << 12
    int disorder_h, hydrogen_type, n_rec_types, n_atom_maps;
    double solpar_q;
    // DS/D1 atoms (hbond 1 or 2) in file order
    int n_h;
    const int *h_index;
    // cell list over the grid box grown by DF_RADIUS, [conf]
    int ncx, ncy, ncz;
    double cell0[3], cell_size;
    const int *cell_start, *cell_atoms;
    // slots: every map except the e map; maps per conformer in the output;
    // slots per (type, bin) row of the vdW table
    int n_slots, n_mm, n_maps_out, tab_stride;
    int need_sol;                // 1: some slot reads the desolvation table (a d map or a desolvation term)
    int need_ang;                // 1: some slot's term uses the directional factors
    int slot_map[DF_MAXS];       // output map index
    int slot_kind[DF_MAXS];      // DK_*
    int slot_tab[DF_MAXS];       // atom-map index of the pair term (-1: none)
    int slot_mm[DF_MAXS];        // min/max register or -1
    int slot_desolv[DF_MAXS];    // 1: receives a desolvation term
    double slot_sp[DF_MAXS], slot_vp[DF_MAXS];
    uint8_t act[DF_MAXS][16];    // [slot][hbond + 8 * disorder]
    double cov_pos[3], cov_half_width, cov_barrier;
    int elec_map;
};

constexpr int DM_TYPE_MASK = 31, DM_HB_SHIFT = 5, DM_REXP_SHIFT = 8;
constexpr int DM_DIS = 1 << 11, DM_SKIP = 1 << 12;

// Interpolation tables, (value, next - value) per bin, in the working
// precision: vdw [n_rec_types][NEINT][tab_stride] (slot s of a row holds the
// table of the slot's atom map, so one pair's slots are one contiguous read),
// sol [NEINT], eps [NDIEL] (dielectric factor * coeff_estat).
template <class R> struct R2 { R v, d; };

struct DiffGrads {
    double *xyz, *q, *rv, *rv2;  // [3N], [N], [3N], [3N] of conformer 0; stride 10N
};

// Per-conformer views of the [conf] arrays.
struct ConfView {
    const double *x, *y, *z, *q, *rv, *rv2;
    const int *cell_start, *cell_atoms;
    DiffGrads g;
};
__host__ __device__ inline ConfView conf_view(const DiffArgs &a, DiffGrads g, int k)
{
    const long long N = a.n_atoms, nc = (long long)a.ncx * a.ncy * a.ncz + 1;
    ConfView v;
    v.x = a.x + k * N; v.y = a.y + k * N; v.z = a.z + k * N; v.q = a.q + k * N;
    v.rv = a.rv + 3 * k * N; v.rv2 = a.rv2 + 3 * k * N;
    v.cell_start = a.cell_start + k * nc;
    v.cell_atoms = a.cell_atoms + k * N;
    const long long go = 10 * k * N;
    v.g.xyz = g.xyz ? g.xyz + go : nullptr;
    v.g.q = g.q ? g.q + go : nullptr;
    v.g.rv = g.rv ? g.rv + go : nullptr;
    v.g.rv2 = g.rv2 ? g.rv2 + go : nullptr;
    return v;
}

cudaError_t launch_closest_h(const DiffArgs &a, int *ch, cudaStream_t s);
// kernels/diff_atoms.cu: atom state rebuilt on the device
cudaError_t launch_split_atoms(long long KN, const double *coord, const double *charge, double *x, double *y,
                               double *z, double *q, int *bad, cudaStream_t s);
cudaError_t launch_bond_vectors(int K, int N, const int *topo, const double *x, const double *y, const double *z,
                                double *rv, double *rv2, cudaStream_t s);
cudaError_t launch_bond_vectors_adj(int K, int N, const int *topo, const double *x, const double *y, const double *z,
                                    const double *grad, double *gx, cudaStream_t s);
cudaError_t launch_cell_lists(const DiffArgs &a, int *cell_of, int *count, cudaStream_t s);
cudaError_t launch_emap_lin(bool fp64, const DiffArgs &a, const void *eps, void *emap, cudaStream_t s);
cudaError_t launch_emap_lin_adj(bool fp64, const DiffArgs &a, const void *eps, const void *g_e, DiffGrads g,
                                cudaStream_t s);
cudaError_t launch_near_lin(bool fp64, const DiffArgs &a, const void *vdw, const void *sol, void *maps,
                            const int *ch, int *mmarg, cudaStream_t s);
cudaError_t launch_near_lin_adj(bool fp64, const DiffArgs &a, const void *vdw, const void *sol, const void *g_maps,
                                const int *ch, const int *mmarg, DiffGrads g, cudaStream_t s);

}  // namespace agb
