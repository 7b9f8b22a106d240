// Per-conformer atom state of the differentiable mode, rebuilt on the device
// from device coordinates: the SoA split, the bond vectors on the frozen bond
// topology (main.cpp:2297-2659 restated for arbitrary coordinates, as the
// host's Job::eval_bond_vectors does), their adjoint, and the cell list the
// short-range kernels walk.
//
// Bond topology: int32 [N][7] = kind, i1, i2, nb, nbr[3] (AG_BOND_* kinds;
// ag_job_bond_topology).  Vector helpers follow main.cpp:3606-3633:
// vect_normalize divides by the nested-hypot length (1e-6 below 1e-6),
// vect_sub_normalize by sqrt of the squared length (1e-6 below 1e-6 squared).
#include <cuda_runtime.h>

#include "autogrid_b200.h"
#include "kernels/diff.h"

namespace agb {

namespace {

constexpr double kZero = 1.0e-6;  // APPROX_ZERO, autocomm.h:72
constexpr int kThreads = 256;

__device__ __forceinline__ void load3(const double *x, const double *y, const double *z, int a, double o[3])
{
    o[0] = x[a];
    o[1] = y[a];
    o[2] = z[a];
}

__device__ __forceinline__ void vnormalize(double v[3])
{
    const double rd = hypot(v[0], hypot(v[1], v[2]));
    const double inv = (rd < kZero) ? 1. / kZero : 1. / rd;
    for (int i = 0; i < 3; i++) v[i] *= inv;
}

__device__ __forceinline__ void vsub_normalize(double o[3], const double a[3], const double b[3])
{
    double rd2 = 0.;
    for (int i = 0; i < 3; i++) {
        o[i] = a[i] - b[i];
        rd2 += o[i] * o[i];
    }
    const double rd = (rd2 < kZero) ? kZero : sqrt(rd2);
    const double inv = 1. / rd;
    for (int i = 0; i < 3; i++) o[i] *= inv;
}

// gv = J^T gy of vnormalize (sub = false) / vsub_normalize (sub = true) at v.
__device__ __forceinline__ void normalize_bwd(const double v[3], const double gy[3], double gv[3], bool sub)
{
    double rd;
    bool below;
    if (sub) {
        const double rd2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        below = rd2 < kZero;
        rd = below ? kZero : sqrt(rd2);
    } else {
        rd = hypot(v[0], hypot(v[1], v[2]));
        below = rd < kZero;
        if (below) rd = kZero;
    }
    if (below) {
        for (int i = 0; i < 3; i++) gv[i] = gy[i] / rd;
        return;
    }
    const double y[3] = {v[0] / rd, v[1] / rd, v[2] / rd};
    const double yg = y[0] * gy[0] + y[1] * gy[1] + y[2] * gy[2];
    for (int i = 0; i < 3; i++) gv[i] = (gy[i] - y[i] * yg) / rd;
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// coord [K][N][3] -> x, y, z [K][N]; charge [K][N] -> q (when given).
// Non-finite input sets *bad.
__global__ void __launch_bounds__(kThreads) k_split_atoms(long long KN, const double *coord, const double *charge,
                                                          double *x, double *y, double *z, double *q, int *bad)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= KN) return;
    const double cx = coord[3 * i], cy = coord[3 * i + 1], cz = coord[3 * i + 2];
    bool ok = isfinite(cx) && isfinite(cy) && isfinite(cz);
    x[i] = cx;
    y[i] = cy;
    z[i] = cz;
    if (charge) {
        const double c = charge[i];
        ok = ok && isfinite(c);
        q[i] = c;
    }
    if (!ok) atomicExch(bad, 1);
}

__global__ void __launch_bounds__(kThreads) k_bond_vectors(int K, int N, const int *topo, const double *X,
                                                           const double *Y, const double *Z, double *RV, double *RV2)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= (long long)K * N) return;
    const int k = (int)(i / N), ia = (int)(i - (long long)k * N);
    const double *x = X + (long long)k * N, *y = Y + (long long)k * N, *z = Z + (long long)k * N;
    double *rv = RV + 3 * i, *rv2 = RV2 + 3 * i;
    const int *t = topo + 7 * ia;
    const int kind = t[0], i1 = t[1], i2 = t[2], nb = t[3];
    double r[3] = {0, 0, 0}, r2[3] = {0, 0, 0}, ca[3], c1[3], c2[3];
    load3(x, y, z, ia, ca);
    switch (kind) {
        case AG_BOND_D1:
            load3(x, y, z, i1, c1);
            for (int d = 0; d < 3; d++) r[d] = ca[d] - c1[d];
            vnormalize(r);
            break;
        case AG_BOND_A2_ONE:
            load3(x, y, z, i1, c1);
            vsub_normalize(r, ca, c1);
            if (i2 >= 0) {
                double dd[3];
                load3(x, y, z, i2, c2);
                for (int d = 0; d < 3; d++) dd[d] = c1[d] - c2[d];
                vnormalize(dd);
                cross3(r, dd, r2);
                vnormalize(r2);
            }
            break;
        case AG_BOND_A2_DIS:
            load3(x, y, z, i1, c1);
            vsub_normalize(r, ca, c1);
            break;
        case AG_BOND_A2_TWO: {
            load3(x, y, z, i1, c1);
            load3(x, y, z, i2, c2);
            vsub_normalize(r2, c2, c1);
            double rdot = 0.;
            for (int d = 0; d < 3; d++) rdot += (ca[d] - c1[d]) * r2[d];
            for (int d = 0; d < 3; d++) r[d] = ca[d] - ((rdot * r2[d]) + c1[d]);
            vnormalize(r);
        } break;
        case AG_BOND_A1: {
            double mean[3] = {0, 0, 0};
            for (int b = 0; b < nb; b++) {
                load3(x, y, z, t[4 + b], c1);
                for (int d = 0; d < 3; d++) mean[d] += (ca[d] - c1[d]) / nb;
            }
            vnormalize(mean);
            for (int d = 0; d < 3; d++) r[d] = -1 * mean[d];
        } break;
        default: break;
    }
    for (int d = 0; d < 3; d++) {
        rv[d] = r[d];
        rv2[d] = r2[d];
    }
}

__device__ __forceinline__ void add3(double *g, int a, const double v[3], double s)
{
    for (int d = 0; d < 3; d++) atomicAdd(g + 3 * (long long)a + d, s * v[d]);
}

// gx [K][3N] += d(rv, rv2)/d(coord)^T (g_rv, g_rv2); g_rv/g_rv2 of conformer
// k start at grad + 10N*k + 4N / + 7N (the adjoint kernels' layout).
__global__ void __launch_bounds__(kThreads) k_bond_vectors_adj(int K, int N, const int *topo, const double *X,
                                                               const double *Y, const double *Z, const double *grad,
                                                               double *gx)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= (long long)K * N) return;
    const int k = (int)(i / N), ia = (int)(i - (long long)k * N);
    const double *x = X + (long long)k * N, *y = Y + (long long)k * N, *z = Z + (long long)k * N;
    const double *grv = grad + 10LL * N * k + 4LL * N + 3LL * ia;
    const double *grv2 = grad + 10LL * N * k + 7LL * N + 3LL * ia;
    double *g = gx + 3LL * N * k;
    const int *t = topo + 7 * ia;
    const int kind = t[0], i1 = t[1], i2 = t[2], nb = t[3];
    double ca[3], c1[3], c2[3];
    load3(x, y, z, ia, ca);
    switch (kind) {
        case AG_BOND_D1: {
            double v[3], gv[3];
            load3(x, y, z, i1, c1);
            for (int d = 0; d < 3; d++) v[d] = ca[d] - c1[d];
            normalize_bwd(v, grv, gv, false);
            add3(g, ia, gv, 1.);
            add3(g, i1, gv, -1.);
        } break;
        case AG_BOND_A2_ONE: {
            double u[3], r[3], g_r[3] = {grv[0], grv[1], grv[2]};
            load3(x, y, z, i1, c1);
            for (int d = 0; d < 3; d++) u[d] = ca[d] - c1[d];
            vsub_normalize(r, ca, c1);
            if (i2 >= 0) {
                double dd[3], dn[3], w[3], gw[3], tt[3], gdn[3], gdd[3];
                load3(x, y, z, i2, c2);
                for (int d = 0; d < 3; d++) dd[d] = dn[d] = c1[d] - c2[d];
                vnormalize(dn);
                cross3(r, dn, w);
                normalize_bwd(w, grv2, gw, false);
                cross3(dn, gw, tt);
                for (int d = 0; d < 3; d++) g_r[d] += tt[d];
                cross3(gw, r, gdn);
                normalize_bwd(dd, gdn, gdd, false);
                add3(g, i1, gdd, 1.);
                add3(g, i2, gdd, -1.);
            }
            double gu[3];
            normalize_bwd(u, g_r, gu, true);
            add3(g, ia, gu, 1.);
            add3(g, i1, gu, -1.);
        } break;
        case AG_BOND_A2_DIS: {
            double u[3], gu[3];
            load3(x, y, z, i1, c1);
            for (int d = 0; d < 3; d++) u[d] = ca[d] - c1[d];
            normalize_bwd(u, grv, gu, true);
            add3(g, ia, gu, 1.);
            add3(g, i1, gu, -1.);
        } break;
        case AG_BOND_A2_TWO: {
            double er[3], e[3], s[3], v[3], gv[3];
            load3(x, y, z, i1, c1);
            load3(x, y, z, i2, c2);
            for (int d = 0; d < 3; d++) {
                er[d] = c2[d] - c1[d];
                s[d] = ca[d] - c1[d];
            }
            vsub_normalize(e, c2, c1);
            double rdot = 0.;
            for (int d = 0; d < 3; d++) rdot += s[d] * e[d];
            for (int d = 0; d < 3; d++) v[d] = ca[d] - ((rdot * e[d]) + c1[d]);
            normalize_bwd(v, grv, gv, false);
            const double egv = e[0] * gv[0] + e[1] * gv[1] + e[2] * gv[2];
            double gs[3], ge[3], ger[3];
            for (int d = 0; d < 3; d++) {
                gs[d] = gv[d] - e[d] * egv;  // v = s - (s.e) e
                ge[d] = grv2[d] - (rdot * gv[d] + egv * s[d]);
            }
            normalize_bwd(er, ge, ger, true);
            add3(g, i2, ger, 1.);
            add3(g, i1, ger, -1.);
            add3(g, ia, gs, 1.);
            add3(g, i1, gs, -1.);
        } break;
        case AG_BOND_A1: {
            if (nb == 0) break;
            double mean[3] = {0, 0, 0}, gm[3], gmean[3];
            for (int b = 0; b < nb; b++) {
                load3(x, y, z, t[4 + b], c1);
                for (int d = 0; d < 3; d++) mean[d] += (ca[d] - c1[d]) / nb;
            }
            for (int d = 0; d < 3; d++) gm[d] = -grv[d];
            normalize_bwd(mean, gm, gmean, false);
            add3(g, ia, gmean, 1.);
            for (int b = 0; b < nb; b++) add3(g, t[4 + b], gmean, -1. / nb);
        } break;
        default: break;
    }
}

// Cell list of every conformer over the grid box grown by DF_RADIUS (cells
// of a.cell_size from a.cell0), atoms of a cell in increasing file index --
// the list the host builds (atoms outside the grown box are left out).
__global__ void __launch_bounds__(kThreads) k_cell_of(DiffArgs a, int *cell_of, int *count)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    const int N = a.n_atoms;
    if (i >= (long long)a.n_conf * N) return;
    const int k = (int)(i / N);
    const long long nc = (long long)a.ncx * a.ncy * a.ncz;
    const double pc[3] = {a.x[i], a.y[i], a.z[i]};
    const int ncs[3] = {a.ncx, a.ncy, a.ncz};
    int c[3];
    for (int d = 0; d < 3; d++) {
        const double u = floor((pc[d] - a.cell0[d]) / a.cell_size);
        if (!(u >= 0 && u < ncs[d])) {
            cell_of[i] = -1;
            return;
        }
        c[d] = (int)u;
    }
    const int cell = c[0] + a.ncx * (c[1] + a.ncy * c[2]);
    cell_of[i] = cell;
    atomicAdd(count + (long long)k * nc + cell, 1);
}

// One CTA per conformer: cell_start[k] = exclusive prefix of count[k]
// (ncells + 1 entries); count[k] becomes the running fill position.
__global__ void __launch_bounds__(1024) k_cell_scan(DiffArgs a, int *count)
{
    __shared__ int part[1024];
    const int k = blockIdx.x;
    const long long nc = (long long)a.ncx * a.ncy * a.ncz;
    int *cnt = count + (long long)k * nc;
    int *start = const_cast<int *>(a.cell_start) + (long long)k * (nc + 1);
    const long long seg = (nc + 1023) / 1024;
    const long long c0 = min(nc, (long long)threadIdx.x * seg), c1 = min(nc, c0 + seg);
    int s = 0;
    for (long long c = c0; c < c1; c++) s += cnt[c];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = part[threadIdx.x] - s;
    for (long long c = c0; c < c1; c++) {
        const int n = cnt[c];
        start[c] = run;
        cnt[c] = run;  // fill cursor
        run += n;
    }
    if (threadIdx.x == 1023) start[nc] = part[1023];
}

__global__ void __launch_bounds__(kThreads) k_cell_fill(DiffArgs a, const int *cell_of, int *cursor)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    const int N = a.n_atoms;
    if (i >= (long long)a.n_conf * N) return;
    const int c = cell_of[i];
    if (c < 0) return;
    const int k = (int)(i / N);
    const long long nc = (long long)a.ncx * a.ncy * a.ncz;
    const int pos = atomicAdd(cursor + (long long)k * nc + c, 1);
    const_cast<int *>(a.cell_atoms)[(long long)k * N + pos] = (int)(i - (long long)k * N);
}

// Insertion sort of each cell's atoms by file index (cells hold a few atoms).
__global__ void __launch_bounds__(kThreads) k_cell_sort(DiffArgs a)
{
    const long long nc = (long long)a.ncx * a.ncy * a.ncz;
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (i >= (long long)a.n_conf * nc) return;
    const int k = (int)(i / nc);
    const long long c = i - (long long)k * nc;
    const int *start = a.cell_start + (long long)k * (nc + 1);
    int *list = const_cast<int *>(a.cell_atoms) + (long long)k * a.n_atoms;
    const int b = start[c], e = start[c + 1];
    for (int p = b + 1; p < e; p++) {
        const int v = list[p];
        int q = p - 1;
        while (q >= b && list[q] > v) {
            list[q + 1] = list[q];
            q--;
        }
        list[q + 1] = v;
    }
}

unsigned blocks_for(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace

cudaError_t launch_split_atoms(long long KN, const double *coord, const double *charge, double *x, double *y,
                               double *z, double *q, int *bad, cudaStream_t s)
{
    if (KN <= 0) return cudaSuccess;
    k_split_atoms<<<blocks_for(KN), kThreads, 0, s>>>(KN, coord, charge, x, y, z, q, bad);
    return cudaGetLastError();
}

cudaError_t launch_bond_vectors(int K, int N, const int *topo, const double *x, const double *y, const double *z,
                                double *rv, double *rv2, cudaStream_t s)
{
    if ((long long)K * N <= 0) return cudaSuccess;
    k_bond_vectors<<<blocks_for((long long)K * N), kThreads, 0, s>>>(K, N, topo, x, y, z, rv, rv2);
    return cudaGetLastError();
}

cudaError_t launch_bond_vectors_adj(int K, int N, const int *topo, const double *x, const double *y, const double *z,
                                    const double *grad, double *gx, cudaStream_t s)
{
    if ((long long)K * N <= 0) return cudaSuccess;
    k_bond_vectors_adj<<<blocks_for((long long)K * N), kThreads, 0, s>>>(K, N, topo, x, y, z, grad, gx);
    return cudaGetLastError();
}

cudaError_t launch_cell_lists(const DiffArgs &a, int *cell_of, int *count, cudaStream_t s)
{
    const long long nc = (long long)a.ncx * a.ncy * a.ncz, KN = (long long)a.n_conf * a.n_atoms;
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int) * (size_t)(nc * a.n_conf), s);
    if (e != cudaSuccess) return e;
    if (KN > 0) k_cell_of<<<blocks_for(KN), kThreads, 0, s>>>(a, cell_of, count);
    k_cell_scan<<<a.n_conf, 1024, 0, s>>>(a, count);
    if (KN > 0) k_cell_fill<<<blocks_for(KN), kThreads, 0, s>>>(a, cell_of, count);
    k_cell_sort<<<blocks_for(nc * a.n_conf), kThreads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace agb
