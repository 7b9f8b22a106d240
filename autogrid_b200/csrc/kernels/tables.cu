// Energy tables on the device (main.cpp:2040-2276, distdepdiel.cpp:30-57),
// restated expression by expression with explicitly rounded FP64 operations
// (no contraction), so they differ from the host's only where CUDA's pow and
// exp differ from the host library's:
//
//   e_vdW_Hb[t][m][k]  cA/r^xA - cB/r^xB at r = k/128 (cA, cB from Rij and
//                      epsij when both are zero), clamped to EINTCLAMP, bin 0
//                      EINTCLAMP, bin NEINT-1 zero, then the +-i_smooth bin
//                      minimum filter (main.cpp:2190-2216); covalent maps
//                      keep zeros;
//   sol_fn[k]          coeff_desolv * exp(-r^2 / (2 sigma^2)), sigma = 3.6,
//                      sol_fn[0] = 0 (main.cpp:2268-2276);
//   r_epsilon_fn[k]    332 / eps(r), eps of Mehler and Solmajer, eps(0) = 1
//                      (main.cpp:1607-1639).
//
// Also the packing a plan needs from tables that are already in device
// memory (the host path in build_plan does the same on the host).
#include <cuda_runtime.h>

#include "autogrid_b200.h"
#include "kernels/tables.h"

namespace agb {

namespace {

constexpr int kThreads = 256;
constexpr double kEintClamp = 100000.;  // autocomm.h:89
constexpr double kApproxZero = 1.0e-6;  // autocomm.h:72
constexpr double kFactor = 332.0;       // main.cpp:561

__device__ __forceinline__ double angstrom(int k) { return __dmul_rn((double)k, 1. / AG_A_DIV); }

// Unsmoothed table of (map m, type t), bin k; sets *bad on the reference's
// fatal conditions (main.cpp:2166-2183).
__global__ void __launch_bounds__(kThreads) k_lj_raw(TableArgs a, float *raw, int *bad)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    const long long n = (long long)a.n_atom_maps * a.n_rec_types * AG_NEINT;
    if (i >= n) return;
    const int k = (int)(i % AG_NEINT);
    const int t = (int)((i / AG_NEINT) % a.n_rec_types);
    const int m = (int)(i / ((long long)AG_NEINT * a.n_rec_types));
    float *tab = raw + ((long long)t * a.n_atom_maps + m) * AG_NEINT;  // [t][m][k]
    if (a.map_is_covalent[m]) {
        tab[k] = 0.f;
        return;
    }
    const int pm = m * a.n_rec_types + t;  // parameters [m][t]
    double cA = a.cA[pm], cB = a.cB[pm];
    const double Rij = a.Rij[pm], epsij = a.epsij[pm];
    const int xA = a.xA[pm], xB = a.xB[pm];
    if (cA == 0 && cB == 0) {
        const double tmpconst = __ddiv_rn(epsij, (double)(xA - xB));
        cA = __dmul_rn(__dmul_rn(tmpconst, pow(Rij, (double)xA)), (double)xB);
        cB = __dmul_rn(__dmul_rn(tmpconst, pow(Rij, (double)xB)), (double)xA);
    }
    if (isnan(cA) || isnan(cB) || xA == 0 || xB == 0) {
        atomicExch(bad, 1);
        return;
    }
    float v;
    if (k == 0) {
        v = (float)kEintClamp;
    } else if (k == AG_NEINT - 1) {
        v = 0.f;
    } else {
        const double r = angstrom(k);
        const double rA = pow(r, (double)xA), rB = pow(r, (double)xB);
        const double e = __dsub_rn(__ddiv_rn(cA, rA), __ddiv_rn(cB, rB));
        v = (float)((kEintClamp < e) ? kEintClamp : e);
    }
    tab[k] = v;
}

// Minimum over bins [k - i_smooth, k + i_smooth] (clipped to the table), as
// main.cpp:2196-2212 takes it, starting from 100000.
__global__ void __launch_bounds__(kThreads) k_lj_smooth(TableArgs a, const float *raw, float *out)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    const long long n = (long long)a.n_atom_maps * a.n_rec_types * AG_NEINT;
    if (i >= n) return;
    const int k = (int)(i % AG_NEINT);
    const long long row = i - k;
    const int m = (int)((i / AG_NEINT) % a.n_atom_maps);
    if (a.i_smooth <= 0 || a.map_is_covalent[m]) {
        out[i] = raw[i];
        return;
    }
    double s = 100000.;
    const int lo = max(0, k - a.i_smooth), hi = min(AG_NEINT, k + a.i_smooth + 1);
    for (int j = lo; j < hi; j++) {
        const double v = (double)raw[row + j];
        s = (s < v) ? s : v;
    }
    out[i] = (float)s;
}

__global__ void __launch_bounds__(kThreads) k_sol_eps(TableArgs a, double *sol_fn, double *r_eps)
{
    const int k = blockIdx.x * kThreads + threadIdx.x;
    if (k >= AG_NDIEL) return;
    const double r = angstrom(k);
    const double sigma = 3.6;
    sol_fn[k] = k == 0 ? 0.0
                       : __dmul_rn(a.coeff_desolv,
                                   exp(__ddiv_rn(-__dmul_rn(r, r), __dmul_rn(2., __dmul_rn(sigma, sigma)))));
    if (r_eps) {
        double eps = 1.0;
        if (k > 0) {
            const double lambda = 0.003627, epsilon0 = 78.4, A = -8.5525, rk = 7.7839;
            const double B = __dsub_rn(epsilon0, A);
            const double lambda_B = __dmul_rn(-lambda, B);
            eps = __dadd_rn(A, __ddiv_rn(B, __dadd_rn(1.0, __dmul_rn(rk, exp(__dmul_rn(lambda_B, r))))));
            if (eps < kApproxZero) eps = 1.0;
        }
        r_eps[k] = __ddiv_rn(kFactor, eps);
    }
}

// Plan tables from device-resident problem tables: vdwT [type][bin][mpad]
// (column c holds map colmap[c], or zeros), far_tab [tab_len + NDIEL] (the
// far kernel's table: zero below FAR_BIN0, bin NDIEL-1 repeated up to
// tab_len; then the whole table) / etab / solf (FP32) and
// reps (FP64, distance-dependent dielectric only).
__global__ void __launch_bounds__(kThreads) k_pack_vdw(const float *e_vdw_hb, int n_rec_types, int n_atom_maps,
                                                       const int *colmap, int mpad, float *vdwT)
{
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    const long long n = (long long)n_rec_types * AG_NEINT * mpad;
    if (i >= n) return;
    const int c = (int)(i % mpad);
    const int b = (int)((i / mpad) % AG_NEINT);
    const int t = (int)(i / ((long long)mpad * AG_NEINT));
    const int m = colmap[c];
    vdwT[i] = m < 0 ? 0.f : e_vdw_hb[((long long)t * n_atom_maps + m) * AG_NEINT + b];
}

__global__ void __launch_bounds__(kThreads) k_pack_lines(const double *sol_fn, const double *r_eps, int dddiel,
                                                         double invdielcal, double coeff_estat, float *far_tab,
                                                         int tab_len, float *etab, float *solf, double *reps)
{
    const int k = blockIdx.x * kThreads + threadIdx.x;
    if (k >= AG_NDIEL && k < tab_len) {  // the far table's extension repeats its last bin
        far_tab[k] = (float)(dddiel ? r_eps[AG_NDIEL - 1] : invdielcal);
        return;
    }
    if (k >= AG_NDIEL) return;
    const double f = dddiel ? r_eps[k] : invdielcal;
    if (reps) reps[k] = dddiel ? r_eps[k] : 0.0;
    if (k < tab_len) far_tab[k] = k < AG_NEINT ? 0.f : (float)f;
    far_tab[tab_len + k] = (float)f;  // the whole table, for the far kernel's bin guard
    etab[k] = (float)__dmul_rn(f, coeff_estat);
    solf[k] = (float)sol_fn[k];
}

unsigned blocks_for(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace

cudaError_t launch_tables_build(const TableArgs &a, float *raw, float *e_vdw_hb, double *sol_fn, double *r_eps,
                                int *bad, cudaStream_t s)
{
    const long long n = (long long)a.n_atom_maps * a.n_rec_types * AG_NEINT;
    if (n > 0) {
        k_lj_raw<<<blocks_for(n), kThreads, 0, s>>>(a, raw, bad);
        k_lj_smooth<<<blocks_for(n), kThreads, 0, s>>>(a, raw, e_vdw_hb);
    }
    k_sol_eps<<<blocks_for(AG_NDIEL), kThreads, 0, s>>>(a, sol_fn, r_eps);
    return cudaGetLastError();
}

cudaError_t launch_pack_tables(const float *e_vdw_hb, int n_rec_types, int n_atom_maps, const int *colmap, int mpad,
                               float *vdwT, const double *sol_fn, const double *r_eps, int dddiel, double invdielcal,
                               double coeff_estat, float *far_tab, int tab_len, float *etab, float *solf,
                               double *reps, cudaStream_t s)
{
    const long long n = (long long)n_rec_types * AG_NEINT * mpad;
    if (n > 0) k_pack_vdw<<<blocks_for(n), kThreads, 0, s>>>(e_vdw_hb, n_rec_types, n_atom_maps, colmap, mpad, vdwT);
    k_pack_lines<<<blocks_for(std::max(AG_NDIEL, tab_len)), kThreads, 0, s>>>(sol_fn, r_eps, dddiel, invdielcal,
                                                                               coeff_estat, far_tab, tab_len, etab,
                                                                               solf, reps);
    return cudaGetLastError();
}

}  // namespace agb
