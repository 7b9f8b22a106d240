// Host-side launchers of the map kernels (defined next to each kernel).
#pragma once
#include <cuda_runtime.h>

#include "agb_device.cuh"
#include "near_params.h"

namespace agb {

struct NearPtrs {
    const float4 *atomA, *atomB;
    const int *meta;
    const float *vdwT;
    int mpad;
    const float *etab, *solf;
    const double *cov_map;
    float *out32;
    double *out64;
    unsigned long long *counters;
};

struct NearSmem {
    float4 pos[NB_CHUNK_MAX], a[NB_CHUNK_MAX], b[NB_CHUNK_MAX];
    int meta[NB_CHUNK_MAX], idx[NB_CHUNK_MAX];
    int hl[NB_CHUNK_MAX], nh;  // staged DS/D1 candidates (slots in this chunk), any order
    // per warp: slots of the staged atoms near that warp's points, in staged order
    unsigned short wl[NB_WARPS_MAX][NB_CHUNK_MAX];
    float wbox[NB_WARPS_MAX][6];  // per warp: its points' box in frame bins (lo xyz, hi xyz)
    float etab[NT_SMALL], sol[NT_SMALL];
    // per thread: the running H-bond min/max of the MM maps (FP32 kernels;
    // in shared memory, out of the pair loop's 80-register budget)
    float hmin[NG_MM][NB_THREADS_MAX], hmax[NG_MM][NB_THREADS_MAX];
    int seg_start[NB_SEGS_MAX], seg_off[NB_SEGS_MAX + 1];
    int tcnt[NB_CHUNK_MAX / 32][32];  // staging by receptor type: per 32-candidate slice and type
    int total;
};

struct NearInst {
    DevProblem p;
    NearGroup g;
    NearPtrs ptr;
};


size_t far_smem_bytes(int tile, int tab_len);
// Dynamic shared-memory limits of the far kernels on the current device.
cudaError_t prepare_far_kernels();
cudaError_t launch_far_bins_debug(const FarArgs &a, const long long *pts, int n_pts, int *used, int *fp32, int *flags,
                                  cudaStream_t s);
cudaError_t launch_emap_far(const FarArgs &a, int n_chunks, int tile, cudaStream_t s, int fz0 = 0, int fz1 = -1);
cudaError_t launch_emap_far_batch(const FarArgs *insts, const long long *unit_begin, int n_inst,
                                  unsigned long long *counter, int tile, int ctas_per_sm, int max_tab_len,
                                  cudaStream_t s);
// The far-field bin fix-up after launch_emap_far (same frames) / the batch kernel.
cudaError_t launch_far_fixup(const FarArgs &a, int n_chunks, cudaStream_t s, int fz0 = 0, int fz1 = -1);
cudaError_t launch_far_fixup_batch(const FarArgs *insts, const long long *unit_begin, int n_inst, long long n_units,
                                   cudaStream_t s);
// Bytes of the edge-bit words of one instance: chunks x frames x words x threads.
size_t far_edge_bits_bytes(int n_chunks, int chunk_atoms, int nframes);
int far_edge_words(int chunk_atoms);
// One instance of the e-map reduction: out[lin] = sum_c partial[c][lin] + out[lin].
struct ReduceInst {
    long long P;
    int n_chunks;
    const float *partial;
    float *out;
};
cudaError_t launch_emap_reduce(const ReduceInst *insts, const long long *begin, int n, long long total,
                               cudaStream_t s);
cudaError_t launch_emap_reduce_range(const ReduceInst &r, long long lin0, long long lin1, cudaStream_t s);
cudaError_t launch_emap_exact(const DevProblem &p, double *emap, cudaStream_t s);
cudaError_t launch_covalent(const DevProblem &p, double *cov, cudaStream_t s);
cudaError_t launch_distance_maps(const DevProblem &p, double cutoff, float *fmap32, float *cmap32, double *fmap64,
                                 double *cmap64, cudaStream_t s);
// 'map_receptor_interior off': collision points of [lin0, lin1) get e = 0 and
// fmap = 1.5, the constriction grid the BH tree's single-precision count
// (any map pointer may be null).
cudaError_t launch_collisions(const DevProblem &p, long long lin0, long long lin1, double cc_cut, float *emap32,
                              float *fmap32, float *cmap32, double *emap64, double *fmap64, double *cmap64,
                              cudaStream_t s);
// Adjoint of the floating grid (dL/d(coord) of the nearest atom of each point),
// added into g_xyz [3N] (FP64); g_fmap [P] in FP32 or FP64.
cudaError_t launch_fmap_adjoint(const DevProblem &p, const void *g_fmap, bool fp64, double *g_xyz, cudaStream_t s);
int near_bricks(const DevProblem &p, int shape);
cudaError_t launch_near(bool exact, const DevProblem &p, const NearGroup &g, const NearPtrs &ptr, int shape,
                        cudaStream_t s, int bz0 = 0, int bz1 = -1);
// max_ng: the most maps any instance's group holds (picks the accumulator count)
cudaError_t launch_near_batch(const NearInst *insts, const long long *unit_begin, int n_inst,
                              unsigned long long *counter, int shape, int ctas_per_sm, int max_ng, cudaStream_t s);
int frames_x(int n1x);
int frames_y(int n1y);
int frames_z(int n1z);

}  // namespace agb
