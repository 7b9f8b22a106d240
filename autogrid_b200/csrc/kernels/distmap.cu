// Distance maps of LOOP 1 (main.cpp:2947-2966): the floating grid (distance
// from each point to the nearest receptor atom, BIG = 1e12 with no atom,
// main.cpp:1882, :2958-2961) and the constriction grid (number of atoms
// within constriction_distance_cutoff, main.cpp:2962-2965).  Both use the
// reference's distance, hypot(dx, hypot(dy, dz)) clamped below at
// APPROX_ZERO, in FP64.  One thread per point; atoms staged through shared
// memory; the squared FP64 distance screens every pair and hypot() is
// evaluated only for the two nearest atoms and for atoms whose squared
// distance lies within 1e-12 of the cutoff, so the reference's comparisons are
// reproduced exactly.
#include "agb_device.cuh"
#include "kernels.h"

namespace agb {

namespace {

constexpr int DM_THREADS = 256;
constexpr double DM_BIG = 1.0e12, DM_APPROX_ZERO = 1.0e-6, DM_REL = 1.0e-12;

__device__ __forceinline__ double ref_dist(double ax, double ay, double az, double cx, double cy, double cz)
{
    double r = hypot(ax - cx, hypot(ay - cy, az - cz));
    return r < DM_APPROX_ZERO ? DM_APPROX_ZERO : r;
}

template <class T>
__global__ void __launch_bounds__(DM_THREADS)
k_distance_maps(DevProblem p, double cutoff, T *__restrict__ fmap, T *__restrict__ cmap)
{
    __shared__ double sx[DM_THREADS], sy[DM_THREADS], sz[DM_THREADS];
    const long long lin = (long long)blockIdx.x * DM_THREADS + threadIdx.x;
    const bool valid = lin < p.P;
    const long long l = valid ? lin : 0;
    const int ix = (int)(l % p.n1x), iy = (int)((l / p.n1x) % p.n1y), iz = (int)(l / ((long long)p.n1x * p.n1y));
    const double cx = (double)(ix - p.nex) * p.spacing, cy = (double)(iy - p.ney) * p.spacing,
                 cz = (double)(iz - p.nez) * p.spacing;
    const double cut2 = cutoff * cutoff;
    double best = 1e300, second = 1e300;
    int ib = -1, is = -1, count = 0;
    for (int a0 = 0; a0 < p.n_atoms; a0 += DM_THREADS) {
        const int na = min(DM_THREADS, p.n_atoms - a0);
        __syncthreads();
        if (threadIdx.x < na) {
            sx[threadIdx.x] = p.x[a0 + threadIdx.x];
            sy[threadIdx.x] = p.y[a0 + threadIdx.x];
            sz[threadIdx.x] = p.z[a0 + threadIdx.x];
        }
        __syncthreads();
        if (!valid) continue;
        for (int j = 0; j < na; j++) {
            const double dx = sx[j] - cx, dy = sy[j] - cy, dz = sz[j] - cz;
            const double s = dx * dx + dy * dy + dz * dz;
            if (fmap) {
                if (s < best) { second = best; is = ib; best = s; ib = a0 + j; }
                else if (s < second) { second = s; is = a0 + j; }
            }
            if (cmap) {
                if (s < cut2 * (1.0 - DM_REL)) count++;
                else if (s <= cut2 * (1.0 + DM_REL) && ref_dist(sx[j], sy[j], sz[j], cx, cy, cz) <= cutoff) count++;
            }
        }
    }
    if (!valid) return;
    if (fmap) {
        double r = DM_BIG;
        if (ib >= 0) r = fmin(r, ref_dist(p.x[ib], p.y[ib], p.z[ib], cx, cy, cz));
        if (is >= 0 && second <= best * (1.0 + DM_REL) + 1e-300)
            r = fmin(r, ref_dist(p.x[is], p.y[is], p.z[is], cx, cy, cz));
        fmap[lin] = (T)r;
    }
    if (cmap) cmap[lin] = (T)count;
}

}  // namespace

cudaError_t launch_distance_maps(const DevProblem &p, double cutoff, float *fmap32, float *cmap32, double *fmap64,
                                 double *cmap64, cudaStream_t s)
{
    if (p.P == 0) return cudaSuccess;
    const unsigned nb = (unsigned)((p.P + DM_THREADS - 1) / DM_THREADS);
    if (fmap64 || cmap64) k_distance_maps<double><<<nb, DM_THREADS, 0, s>>>(p, cutoff, fmap64, cmap64);
    else k_distance_maps<float><<<nb, DM_THREADS, 0, s>>>(p, cutoff, fmap32, cmap32);
    return cudaGetLastError();
}

}  // namespace agb
