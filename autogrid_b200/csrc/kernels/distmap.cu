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

// Adjoint of the floating grid: r_min(p) = |x_a - c_p| for the nearest atom a
// (lowest index among equals), so dL/dx_a += g_p (x_a - c_p) / r.  Points with
// no atom (r_min = BIG) or an atom closer than APPROX_ZERO (clamped) give none.
template <class T>
__global__ void __launch_bounds__(DM_THREADS) k_fmap_adjoint(DevProblem p, const T *__restrict__ g_fmap,
                                                             double *__restrict__ g_xyz)
{
    __shared__ double sx[DM_THREADS], sy[DM_THREADS], sz[DM_THREADS];
    const long long lin = (long long)blockIdx.x * DM_THREADS + threadIdx.x;
    const bool valid = lin < p.P;
    const long long l = valid ? lin : 0;
    const int ix = (int)(l % p.n1x), iy = (int)((l / p.n1x) % p.n1y), iz = (int)(l / ((long long)p.n1x * p.n1y));
    const double cx = (double)(ix - p.nex) * p.spacing, cy = (double)(iy - p.ney) * p.spacing,
                 cz = (double)(iz - p.nez) * p.spacing;
    double best = 1e300;
    int ib = -1;
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
            if (s < best) { best = s; ib = a0 + j; }
        }
    }
    if (!valid || ib < 0) return;
    const double g = (double)g_fmap[lin];
    const double dx = p.x[ib] - cx, dy = p.y[ib] - cy, dz = p.z[ib] - cz;
    const double r = ref_dist(p.x[ib], p.y[ib], p.z[ib], cx, cy, cz);
    if (g == 0.0 || !(r > DM_APPROX_ZERO)) return;
    atomicAdd(g_xyz + 3 * ib, g * dx / r);
    atomicAdd(g_xyz + 3 * ib + 1, g * dy / r);
    atomicAdd(g_xyz + 3 * ib + 2, g * dz / r);
}

// The BH tree's close-atom test in single precision (bhtree.cpp:338-366):
// float differences of the float grid point and float atom coordinates, each
// within the cutoff, and their float squared sum (left to right, no fused
// multiply-add) not above the float squared cutoff.
__device__ __forceinline__ bool bh_close(float px, float py, float pz, float ax, float ay, float az, float cut,
                                         float cut2)
{
    const float d0 = __fsub_rn(px, ax);
    if (d0 > cut || d0 < -cut) return false;
    const float d1 = __fsub_rn(py, ay);
    if (d1 > cut || d1 < -cut) return false;
    const float d2 = __fsub_rn(pz, az);
    if (d2 > cut || d2 < -cut) return false;
    const float D = __fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)), __fmul_rn(d2, d2));
    return !(D > cut2);
}

// 'map_receptor_interior off' (main.cpp:2893-2927, the USE_BHTREE build):
// points [lin0, lin1) with an atom within BH_COLLISION_DIST are collisions --
// e map 0, floating grid BH_COLLISION_DIST -- and the constriction grid is
// the BH tree's count within its cutoff.  Atoms come from the cell list when
// the largest cutoff is within the cell list's reach (8 A), else from all atoms.
constexpr float BH_COLLISION_DIST = 1.5f;  // main.cpp:346
template <class T>
__global__ void __launch_bounds__(DM_THREADS) k_collisions(DevProblem p, long long lin0, long long lin1, float cc_cut,
                                                           T *__restrict__ emap, T *__restrict__ fmap,
                                                           T *__restrict__ cmap)
{
    const long long lin = lin0 + (long long)blockIdx.x * DM_THREADS + threadIdx.x;
    if (lin >= lin1) return;
    const int ix = (int)(lin % p.n1x), iy = (int)((lin / p.n1x) % p.n1y), iz = (int)(lin / ((long long)p.n1x * p.n1y));
    const double c[3] = {(double)(ix - p.nex) * p.spacing, (double)(iy - p.ney) * p.spacing,
                         (double)(iz - p.nez) * p.spacing};
    const float px = (float)c[0], py = (float)c[1], pz = (float)c[2];  // fcc, main.cpp:2860
    const float bh = BH_COLLISION_DIST, bh2 = __fmul_rn(bh, bh);
    const float cc2 = __fmul_rn(cc_cut, cc_cut);
    const bool want_count = cmap != nullptr;
    const float reach = want_count ? fmaxf(bh, cc_cut) : bh;
    bool hit = false;
    int count = 0;
    auto visit = [&](int a) {
        const float ax = (float)p.x[a], ay = (float)p.y[a], az = (float)p.z[a];
        if (!hit && bh_close(px, py, pz, ax, ay, az, bh, bh2)) hit = true;
        if (want_count && bh_close(px, py, pz, ax, ay, az, cc_cut, cc2)) count++;
    };
    if ((double)reach <= 8.0) {
        int lo[3], hi[3];
        const int nc[3] = {p.ncx, p.ncy, p.ncz};
        for (int i = 0; i < 3; i++) {
            lo[i] = max(0, min(nc[i] - 1, (int)floor((c[i] - (double)reach - 1e-3 - p.cell0[i]) / p.cell_size)));
            hi[i] = max(0, min(nc[i] - 1, (int)floor((c[i] + (double)reach + 1e-3 - p.cell0[i]) / p.cell_size)));
        }
        for (int cz = lo[2]; cz <= hi[2]; cz++)
            for (int cy = lo[1]; cy <= hi[1]; cy++) {
                const int c0 = (cz * p.ncy + cy) * p.ncx;
                for (int k = p.cell_start[c0 + lo[0]]; k < p.cell_start[c0 + hi[0] + 1]; k++) visit(p.cell_atoms[k]);
            }
    } else {
        for (int a = 0; a < p.n_atoms; a++) visit(a);
    }
    if (hit) {
        if (emap) emap[lin] = (T)0;
        if (fmap) fmap[lin] = (T)BH_COLLISION_DIST;
    }
    if (want_count) cmap[lin] = (T)count;
}

}  // namespace

cudaError_t launch_collisions(const DevProblem &p, long long lin0, long long lin1, double cc_cut, float *emap32,
                              float *fmap32, float *cmap32, double *emap64, double *fmap64, double *cmap64,
                              cudaStream_t s)
{
    if (lin1 <= lin0) return cudaSuccess;
    const unsigned nb = (unsigned)((lin1 - lin0 + DM_THREADS - 1) / DM_THREADS);
    if (emap64 || fmap64 || cmap64)
        k_collisions<double><<<nb, DM_THREADS, 0, s>>>(p, lin0, lin1, (float)cc_cut, emap64, fmap64, cmap64);
    else
        k_collisions<float><<<nb, DM_THREADS, 0, s>>>(p, lin0, lin1, (float)cc_cut, emap32, fmap32, cmap32);
    return cudaGetLastError();
}

cudaError_t launch_fmap_adjoint(const DevProblem &p, const void *g_fmap, bool fp64, double *g_xyz, cudaStream_t s)
{
    if (p.P == 0 || p.n_atoms == 0) return cudaSuccess;
    const unsigned nb = (unsigned)((p.P + DM_THREADS - 1) / DM_THREADS);
    if (fp64) k_fmap_adjoint<double><<<nb, DM_THREADS, 0, s>>>(p, (const double *)g_fmap, g_xyz);
    else k_fmap_adjoint<float><<<nb, DM_THREADS, 0, s>>>(p, (const float *)g_fmap, g_xyz);
    return cudaGetLastError();
}

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
