// Differentiable mode, electrostatic map: LOOP 1 of main.cpp:2940-2982 with
// the dielectric table read by linear interpolation (kernels/diff.h):
//     e(p) = sum_a q_a F(r_pa),   F(r) = T(A_DIV r) / max(r, 0.5),
// T the table of eps factor * coeff_estat, constant past its last bin.
//   k_emap_lin<R>      forward: one thread per point, atoms staged through
//                      shared memory, the table resident in shared memory;
//   k_emap_lin_adj<R>  adjoint: one thread per atom, points (with dL/de) staged
//                      through shared memory,
//                        dL/dq_a = sum_p g(p) F(r),
//                        dL/dx_a = sum_p g(p) q_a F'(r) (x_a - x_p) / r.
// Algorithmic cost: one pair term per (point, atom), one reciprocal square root
// each (rsqrt.approx in FP32, IEEE sqrt and division in the FP64 twin).
#include "agb_device.cuh"
#include "diff.h"

namespace agb {

namespace {

constexpr int EL_THREADS = 256, EL_TILE = 256;

template <class R> struct Vec4;
template <> struct Vec4<float> { using T = float4; };
template <> struct Vec4<double> { using T = double4; };

// Table value and slope at x = A_DIV r, and 1/max(r, 0.5), from r^2.
__device__ __forceinline__ void lin_eval(const R2<float> *tab, float r2, float &T, float &slope, float &rs)
{
    r2 = fmaxf(r2, 1.0e-12f);
    rs = rsqrt_approx(r2);
    const float x = r2 * rs * (float)AG_A_DIV;
    const float xb = __fadd_rz(x, 8388608.0f);  // 2^23: the low mantissa bits hold floor(x)
    const int b = min(__float_as_int(xb) - 0x4B000000, AG_NDIEL - 1);
    const float fx = x - (xb - 8388608.0f);
    const R2<float> e = tab[b];
    T = fmaf(fx, e.d, e.v);
    slope = e.d * (float)AG_A_DIV;
}
__device__ __forceinline__ void lin_eval(const R2<double> *tab, double r2, double &T, double &slope, double &rs)
{
    double r = sqrt(r2);
    if (r < 1.0e-6) r = 1.0e-6;
    rs = 1.0 / r;
    const double x = r * (double)AG_A_DIV;
    int b = (int)x;
    b = b < AG_NDIEL - 1 ? b : AG_NDIEL - 1;
    const R2<double> e = tab[b];
    T = e.v + (x - (double)b) * e.d;
    slope = e.d * (double)AG_A_DIV;
}

template <class R> __device__ __forceinline__ R point_coord(int i, int ne, double spacing)
{
    return (R)((double)(i - ne) * spacing);
}

template <class R>
__global__ void __launch_bounds__(EL_THREADS) k_emap_lin(DiffArgs a, const R2<R> *__restrict__ gtab, R *__restrict__ emap)
{
    using V4 = typename Vec4<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2<R> *s_tab = reinterpret_cast<R2<R> *>(smem_raw);
    V4 *s_atom = reinterpret_cast<V4 *>(smem_raw + sizeof(R2<R>) * AG_NDIEL);
    for (int i = threadIdx.x; i < AG_NDIEL; i += EL_THREADS) s_tab[i] = gtab[i];
    const ConfView v = conf_view(a, DiffGrads{}, blockIdx.y);  // blockIdx.y: conformer
    emap += (long long)blockIdx.y * a.n_maps_out * a.P;

    const long long lin = (long long)blockIdx.x * EL_THREADS + threadIdx.x;
    const bool valid = lin < a.P;
    const long long l = valid ? lin : 0;
    const int ix = (int)(l % a.n1x), iy = (int)((l / a.n1x) % a.n1y), iz = (int)(l / ((long long)a.n1x * a.n1y));
    const R cx = point_coord<R>(ix, a.nex, a.spacing), cy = point_coord<R>(iy, a.ney, a.spacing),
            cz = point_coord<R>(iz, a.nez, a.spacing);
    R e = 0;
    for (int a0 = 0; a0 < a.n_atoms; a0 += EL_TILE) {
        const int na = min(EL_TILE, a.n_atoms - a0);
        __syncthreads();
        for (int i = threadIdx.x; i < na; i += EL_THREADS) {
            V4 t;
            t.x = (R)v.x[a0 + i]; t.y = (R)v.y[a0 + i]; t.z = (R)v.z[a0 + i]; t.w = (R)v.q[a0 + i];
            s_atom[i] = t;
        }
        __syncthreads();
        R acc = 0;
#pragma unroll 4
        for (int i = 0; i < na; i++) {
            const V4 at = s_atom[i];
            const R dx = at.x - cx, dy = at.y - cy, dz = at.z - cz;
            R T, slope, rs;
            lin_eval(s_tab, dx * dx + dy * dy + dz * dz, T, slope, rs);
            acc += at.w * (T * (rs < (R)2 ? rs : (R)2));
        }
        e += acc;
    }
    if (valid) emap[lin] = e;
}

template <class R>
__global__ void __launch_bounds__(EL_THREADS)
k_emap_lin_adj(DiffArgs a, const R2<R> *__restrict__ gtab, const R *__restrict__ g_e, DiffGrads g_all,
               int points_per_block)
{
    using V4 = typename Vec4<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2<R> *s_tab = reinterpret_cast<R2<R> *>(smem_raw);
    V4 *s_pt = reinterpret_cast<V4 *>(smem_raw + sizeof(R2<R>) * AG_NDIEL);
    for (int i = threadIdx.x; i < AG_NDIEL; i += EL_THREADS) s_tab[i] = gtab[i];
    const ConfView cv = conf_view(a, g_all, blockIdx.z);  // blockIdx.z: conformer
    const DiffGrads g = cv.g;
    g_e += (long long)blockIdx.z * a.n_maps_out * a.P;

    const int at = blockIdx.x * EL_THREADS + threadIdx.x;
    const bool valid = at < a.n_atoms;
    const R xa = valid ? (R)cv.x[at] : (R)0, ya = valid ? (R)cv.y[at] : (R)0, za = valid ? (R)cv.z[at] : (R)0;
    const R qa = valid ? (R)cv.q[at] : (R)0;
    R gx = 0, gy = 0, gz = 0, gq = 0;
    const long long p_begin = (long long)blockIdx.y * points_per_block;
    const long long p_end = min(a.P, p_begin + points_per_block);
    for (long long p0 = p_begin; p0 < p_end; p0 += EL_TILE) {
        const int np = (int)min((long long)EL_TILE, p_end - p0);
        __syncthreads();
        for (int i = threadIdx.x; i < np; i += EL_THREADS) {
            const long long lin = p0 + i;
            const int ix = (int)(lin % a.n1x), iy = (int)((lin / a.n1x) % a.n1y),
                      iz = (int)(lin / ((long long)a.n1x * a.n1y));
            V4 v;
            v.x = point_coord<R>(ix, a.nex, a.spacing);
            v.y = point_coord<R>(iy, a.ney, a.spacing);
            v.z = point_coord<R>(iz, a.nez, a.spacing);
            v.w = g_e[lin];
            s_pt[i] = v;
        }
        __syncthreads();
        R ax = 0, ay = 0, az = 0, aq = 0;
#pragma unroll 4
        for (int i = 0; i < np; i++) {
            const V4 pt = s_pt[i];
            const R dx = xa - pt.x, dy = ya - pt.y, dz = za - pt.z;
            R T, slope, rs;
            lin_eval(s_tab, dx * dx + dy * dy + dz * dz, T, slope, rs);
            const bool outer = rs < (R)2;  // r > 0.5
            const R F = outer ? T * rs : T * (R)2;
            const R dF = outer ? (slope - T * rs) * rs : slope * (R)2;  // dF/dr
            aq += pt.w * F;
            const R s = pt.w * dF * rs;
            ax += s * dx; ay += s * dy; az += s * dz;
        }
        gx += ax; gy += ay; gz += az; gq += aq;
    }
    if (valid) {
        atomicAdd(g.xyz + 3 * at, (double)(gx * qa));
        atomicAdd(g.xyz + 3 * at + 1, (double)(gy * qa));
        atomicAdd(g.xyz + 3 * at + 2, (double)(gz * qa));
        atomicAdd(g.q + at, (double)gq);
    }
}

template <class R> size_t emap_smem() { return sizeof(R2<R>) * AG_NDIEL + sizeof(typename Vec4<R>::T) * EL_TILE; }

template <class R> cudaError_t set_smem(const void *fn)
{
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)emap_smem<R>());
}

}  // namespace

cudaError_t launch_emap_lin(bool fp64, const DiffArgs &a, const void *eps, void *emap, cudaStream_t s)
{
    if (a.P == 0) return cudaSuccess;
    const dim3 nb((unsigned)((a.P + EL_THREADS - 1) / EL_THREADS), (unsigned)a.n_conf);
    cudaError_t e;
    if (fp64) {
        if ((e = set_smem<double>((const void *)k_emap_lin<double>)) != cudaSuccess) return e;
        k_emap_lin<double><<<nb, EL_THREADS, emap_smem<double>(), s>>>(a, (const R2<double> *)eps, (double *)emap);
    } else {
        if ((e = set_smem<float>((const void *)k_emap_lin<float>)) != cudaSuccess) return e;
        k_emap_lin<float><<<nb, EL_THREADS, emap_smem<float>(), s>>>(a, (const R2<float> *)eps, (float *)emap);
    }
    return cudaGetLastError();
}

cudaError_t launch_emap_lin_adj(bool fp64, const DiffArgs &a, const void *eps, const void *g_e, DiffGrads g,
                                cudaStream_t s)
{
    if (a.n_atoms == 0 || a.P == 0) return cudaSuccess;
    // about four blocks per SM over (atom blocks x point ranges)
    const int atom_blocks = (a.n_atoms + EL_THREADS - 1) / EL_THREADS;
    long long ranges = (4LL * current_device_sms() + atom_blocks - 1) / atom_blocks;
    long long ppb = (a.P + ranges - 1) / ranges;
    ppb = ((ppb + EL_TILE - 1) / EL_TILE) * EL_TILE;
    if (ppb < EL_TILE) ppb = EL_TILE;
    ranges = (a.P + ppb - 1) / ppb;
    dim3 grid((unsigned)atom_blocks, (unsigned)ranges, (unsigned)a.n_conf);
    cudaError_t e;
    if (fp64) {
        if ((e = set_smem<double>((const void *)k_emap_lin_adj<double>)) != cudaSuccess) return e;
        k_emap_lin_adj<double><<<grid, EL_THREADS, emap_smem<double>(), s>>>(a, (const R2<double> *)eps,
                                                                            (const double *)g_e, g, (int)ppb);
    } else {
        if ((e = set_smem<float>((const void *)k_emap_lin_adj<float>)) != cudaSuccess) return e;
        k_emap_lin_adj<float><<<grid, EL_THREADS, emap_smem<float>(), s>>>(a, (const R2<float> *)eps,
                                                                          (const float *)g_e, g, (int)ppb);
    }
    return cudaGetLastError();
}

}  // namespace agb
