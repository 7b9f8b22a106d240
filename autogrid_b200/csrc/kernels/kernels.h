// Host-side launchers of the map kernels (defined next to each kernel).
#pragma once
#include <cuda_runtime.h>

#include "agb_device.cuh"
#include "near_params.h"

namespace agb {

cudaError_t launch_emap_far(const double *ax128, const double *ay128, const double *az128, const float *qw,
                            int n_atoms, int chunk_atoms, int n_chunks, const float *far_tab,
                            double spacing_adiv, int n1x, int n1y, int n1z, int nex, int ney, int nez,
                            long long P, float *partial, cudaStream_t s);
cudaError_t launch_emap_exact(const DevProblem &p, double *emap, cudaStream_t s);
cudaError_t launch_covalent(const DevProblem &p, double *cov, cudaStream_t s);
cudaError_t launch_near(bool exact, const DevProblem &p, const NearGroup &g, const float4 *atomA,
                        const float4 *atomB, const int *meta, const float *vdwT, int mpad, const float *etab,
                        const float *solf, const double *cov_map, float *out32, double *out64,
                        unsigned long long *counters, cudaStream_t s);
int frames_x(int n1x);
int frames_y(int n1y);
int frames_z(int n1z);

}  // namespace agb
