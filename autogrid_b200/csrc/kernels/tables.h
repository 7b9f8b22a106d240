// Launchers of the energy-table kernels (kernels/tables.cu).
#pragma once
#include <cuda_runtime.h>

namespace agb {

// Device pointers; parameters are [n_atom_maps][n_rec_types].
struct TableArgs {
    int n_rec_types, n_atom_maps;
    const double *cA, *cB, *Rij, *epsij;
    const int *xA, *xB, *map_is_covalent;
    int i_smooth;          // (int)(r_smooth * A_DIV / 2), main.cpp:2190
    double coeff_desolv;
};

// e_vdw_hb [n_rec_types][n_atom_maps][NEINT] (raw: scratch of the same size),
// sol_fn [NDIEL], r_eps [NDIEL] (NULL: constant dielectric); *bad = 1 on a
// fatal parameter (NaN coefficient or zero exponent).
cudaError_t launch_tables_build(const TableArgs &a, float *raw, float *e_vdw_hb, double *sol_fn, double *r_eps,
                                int *bad, cudaStream_t s);
// Plan tables from device-resident problem tables (colmap [mpad]: map of each
// vdW column, -1 for none).
cudaError_t launch_pack_tables(const float *e_vdw_hb, int n_rec_types, int n_atom_maps, const int *colmap, int mpad,
                               float *vdwT, const double *sol_fn, const double *r_eps, int dddiel, double invdielcal,
                               double coeff_estat, float *far_tab, int tab_len, float *etab, float *solf,
                               double *reps, cudaStream_t s);

}  // namespace agb
