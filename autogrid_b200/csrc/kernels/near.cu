// Near-field kernels: everything of the reference grid loop except the
// far-field electrostatics.
//
//   k_near<EXACT> one thread per grid point, bricks of 8x8x4 points.  Candidate
//                atoms come from a cell list (cells of AGB_CELL A over the box
//                grown by 8.05 A) and are staged through shared memory.
//                Per pair: short-range AD4 terms of LOOP 2 (main.cpp:3030-3404),
//                the d map, and (FP32 path only) the near part of the e map,
//                i.e. the pairs the far-field kernel leaves out.
//       EXACT=true : FP64 twin, every quantity in FP64 exactly as the reference.
//       EXACT=false: FP32 production path.  Distances come from the same
//                canonical frame-relative FP32 arithmetic as the far-field
//                kernel.  Whenever an FP32 quantity lies within its error bound
//                of a discontinuity of the reference (table-bin edge, the
//                8 A cutoff, the cos=0 branch of the D1 and A2 factors, a
//                disordered-hydrogen bin edge) the pair is re-evaluated in FP64
//                with the reference formulas, so table bins equal the FP64
//                reference's.
//   Desolvation is factored: sum_a sol(r)(sp_m vol_a + (solpar_a+qasp|q_a|) vp_m)
//   = sp_m*D1 + vp_m*D2 with D1 = sum vol_a sol, D2 = sum (solpar_a+qasp|q_a|) sol,
//   and the d map is qasp*D1 (main.cpp:3381-3404).
#include <algorithm>
#include <type_traits>

#include "kernels.h"

namespace agb {

constexpr int NB_THREADS = 256;   // one thread per brick point (brick shape is a template parameter)
#ifndef NEAR_MIN_CTAS
#define NEAR_MIN_CTAS 3              // resident CTAs per SM the register allocation targets
#endif
constexpr int NB_CHUNK = NB_CHUNK_MAX;   // candidates staged at once (most bricks need one chunk)
constexpr int NB_SEGS = NB_SEGS_MAX;
constexpr float GUARD_BIN = 2.0e-3f;   // bins: > 3x the FP32 distance error bound
constexpr float GUARD_COS = 5.0e-5f;
constexpr double APPROX_ZERO_D = 1.0e-6;
constexpr double PI_D = 3.14159265358979323846;

// ------------------------------------------------------------ pair state ---
template <class R>
struct PairQ {
    int ad4_in;   // inside 8 A and not a skipped disordered hydrogen
    int bin;      // (int)(r*A_DIV), unclamped
    int bin_e;    // LOOP 1 bin (nested hypot), unclamped
    int ih;       // disordered-hydrogen row bin, clamped to [0, NEINT-1]
    R r, inv_rmax, racc, rdon, Hramp;
};

// FP64, expression-for-expression restatement of main.cpp:3037-3272 for one
// (point, atom) pair.  Explicit _rn intrinsics keep nvcc from contracting.
// The distance part: LOOP 2's distance, cutoff and bins (main.cpp:3037-3046,
// :3309-3311) and LOOP 1's nested-hypot distance and 1/max(r, 0.5)
// (main.cpp:2951-2956).  Returns the pair vector and r.
template <class R>
__device__ __forceinline__ void dist_exact(const DevProblem &p, int ia, double cx, double cy, double cz, PairQ<R> &o,
                                           double &d0, double &d1, double &d2, double &r_out)
{
    d0 = __dsub_rn(p.x[ia], cx); d1 = __dsub_rn(p.y[ia], cy); d2 = __dsub_rn(p.z[ia], cz);
    double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
    double re = hypot(d0, hypot(d1, d2));
    o.ad4_in = !(r > AG_NBC);
    if (p.disorder_h && p.disorder[ia] && p.type[ia] == p.hydrogen_type) o.ad4_in = 0;
    if (r < APPROX_ZERO_D) r = APPROX_ZERO_D;
    if (re < APPROX_ZERO_D) re = APPROX_ZERO_D;
    o.r = (R)r;
    o.inv_rmax = (R)__ddiv_rn(1.0, re > 0.5 ? re : 0.5);
    o.bin = __double2int_rz(__dmul_rn(r, (double)AG_A_DIV));
    o.bin_e = __double2int_rz(__dmul_rn(re, (double)AG_A_DIV));
    int ih = __double2int_rz(__dmul_rn(__dsub_rn(r, 1.10), (double)AG_A_DIV));
    ih = ih < 0 ? 0 : ih;
    o.ih = ih > AG_NEINT - 1 ? AG_NEINT - 1 : ih;
    r_out = r;
}

// Distance part only, for FP32 pairs whose distance lies within its error
// bound of a bin edge; the directional factors stay FP32.
__device__ __noinline__ void dist_exact_f(const DevProblem &p, int ia, double cx, double cy, double cz,
                                          PairQ<float> &o)
{
    double d0, d1, d2, r;
    dist_exact(p, ia, cx, cy, cz, o, d0, d1, d2, r);
}

__device__ __noinline__ void pair_exact(const DevProblem &p, int ia, double cx, double cy, double cz,
                                        int ch, PairQ<double> &o)
{
    double d0, d1, d2, r;
    dist_exact(p, ia, cx, cy, cz, o, d0, d1, d2, r);
    o.racc = 1.0; o.rdon = 1.0; o.Hramp = 1.0;
    const double inv_r = __ddiv_rn(1.0, r);
    const double dn0 = __dmul_rn(d0, inv_r), dn1 = __dmul_rn(d1, inv_r), dn2 = __dmul_rn(d2, inv_r);
    const int hb = p.hbond[ia];
    const double *rv = p.rv + 3 * (size_t)ia;
    const double PI_halved = PI_D / 2.;
    auto negdot = [&](const double *v) {
        double c = 0.;
        c = __dsub_rn(c, __dmul_rn(dn0, v[0]));
        c = __dsub_rn(c, __dmul_rn(dn1, v[1]));
        c = __dsub_rn(c, __dmul_rn(dn2, v[2]));
        return c;
    };
    if (hb == 2) {
        const double cos_theta = negdot(rv);
        if (cos_theta <= 0.) {
            o.racc = 0.;
        } else {
            const int e = p.rexp[ia];
            if (e == 2) o.racc = __dmul_rn(cos_theta, cos_theta);
            else if (e == 4) { const double t = __dmul_rn(cos_theta, cos_theta); o.racc = __dmul_rn(t, t); }
            else o.racc = cos_theta;
            if (ia == ch || ch < 0) {  // ch < 0 only when no ligand map needs Hramp
                o.Hramp = 1.;
            } else {
                const double *rh = p.rv + 3 * (size_t)ch;
                double ct = 0.;
                ct = __dadd_rn(ct, __dmul_rn(rh[0], rv[0]));
                ct = __dadd_rn(ct, __dmul_rn(rh[1], rv[1]));
                ct = __dadd_rn(ct, __dmul_rn(rh[2], rv[2]));
                ct = ct < 1.0 ? ct : 1.0;
                ct = ct > -1.0 ? ct : -1.0;
                const double theta = acos(ct);
                o.Hramp = __dsub_rn(0.5, __dmul_rn(0.5, cos(__ddiv_rn(__dmul_rn(theta, 120.), 90.))));
            }
        }
    } else if (hb == 4) {
        const double cos_theta = negdot(rv);
        o.rdon = (cos_theta <= 0.) ? 0. : __dmul_rn(cos_theta, cos_theta);
    } else if (hb == 5 && !p.disorder[ia]) {
        const double *rv2 = p.rv2 + 3 * (size_t)ia;
        const double cos_theta = negdot(rv);
        double t0 = 0.;
        t0 = __dadd_rn(t0, __dmul_rn(dn0, rv2[0]));
        t0 = __dadd_rn(t0, __dmul_rn(dn1, rv2[1]));
        t0 = __dadd_rn(t0, __dmul_rn(dn2, rv2[2]));
        if (t0 > 1.) t0 = 1.; else if (t0 < -1.) t0 = -1.;
        t0 = __dsub_rn(PI_halved, acos(t0));
        const double c0 = __dsub_rn(__dmul_rn(dn1, rv2[2]), __dmul_rn(dn2, rv2[1]));
        const double c1 = __dsub_rn(__dmul_rn(dn2, rv2[0]), __dmul_rn(dn0, rv2[2]));
        const double c2 = __dsub_rn(__dmul_rn(dn0, rv2[1]), __dmul_rn(dn1, rv2[0]));
        double rd2 = __dadd_rn(__dadd_rn(__dmul_rn(c0, c0), __dmul_rn(c1, c1)), __dmul_rn(c2, c2));
        if (rd2 < APPROX_ZERO_D) rd2 = APPROX_ZERO_D;
        const double inv_rd = __ddiv_rn(1.0, __dsqrt_rn(rd2));
        double ti = 0.;
        ti = __dadd_rn(ti, __dmul_rn(__dmul_rn(c0, inv_rd), rv[0]));
        ti = __dadd_rn(ti, __dmul_rn(__dmul_rn(c1, inv_rd), rv[1]));
        ti = __dadd_rn(ti, __dmul_rn(__dmul_rn(c2, inv_rd), rv[2]));
        o.rdon = 0.;
        if (cos_theta >= 0.) {
            if (ti > 1.) ti = 1.; else if (ti < -1.) ti = -1.;
            ti = __dsub_rn(acos(ti), PI_halved);
            if (ti < 0.) ti = -ti;
            o.rdon = __dmul_rn(__dadd_rn(0.9, __dmul_rn(0.1, sin(__dadd_rn(ti, ti)))), cos(t0));
        } else if (cos_theta >= -0.34202) {
            const double b = __dsub_rn(0.116978, __dmul_rn(cos_theta, cos_theta));
            o.rdon = __dmul_rn(__dmul_rn(562.25, pow(b, 3.)), cos(t0));
        }
    } else if (p.disorder[ia] && hb == 5) {
        double cos_theta = negdot(rv);
        if (cos_theta > 1.) cos_theta = 1.; else if (cos_theta < -1.) cos_theta = -1.;
        const double theta = acos(cos_theta);
        o.racc = 0.; o.rdon = 0.;
        if (theta <= 1.24791 + PI_halved) {
            o.rdon = pow(cos(__dsub_rn(theta, 1.24791)), 4.);
            o.racc = o.rdon;
        }
    }
}

// Per-atom metadata packed for shared memory (built by the host, capi.cu).
constexpr int META_TYPE_MASK = 31;          // bits 0-4   receptor type
constexpr int META_HB_SHIFT = 5;            // bits 5-7   hbond class
constexpr int META_REXP_SHIFT = 8;          // bits 8-10  rexp
constexpr int META_DIS = 1 << 11;           // disorder flag
constexpr int META_RVZERO = 1 << 12;        // bond vector exactly zero
constexpr int META_SKIP_AD4 = 1 << 13;      // disordered hydrogen skipped by LOOP 2 (main.cpp:3052)

// FP32 distance quantities from the canonical frame-relative distance t (in
// bins).  Returns false when t (or the disordered-hydrogen row bin) lies
// within its error bound of a bin edge (the 8 A cutoff is bin 1024); the
// caller then takes the distance part from dist_exact_f().
__device__ __forceinline__ bool dist_fast(int meta, float t, float rs, PairQ<float> &o)
{
    const float tf = floorf(t);
    if (t - tf < GUARD_BIN || (tf + 1.f) - t < GUARD_BIN || t < 1.0f) return false;
    o.bin = (int)tf;
    o.bin_e = o.bin;
    o.ad4_in = (t < FAR_T0) && !(meta & META_SKIP_AD4);  // t is not within GUARD_BIN of 1024: equals r <= 8
    o.r = t * (1.0f / AG_A_DIV);
    o.inv_rmax = fminf((float)AG_A_DIV * rs, 2.0f);
    o.ih = 0;
    if (o.ad4_in && (meta & META_DIS)) {
        const float xh = t - 140.8f;  // (r - 1.10) * A_DIV
        if (xh > 0.5f) {
            const float xf = floorf(xh);
            if (xh - xf < GUARD_BIN || (xf + 1.f) - xh < GUARD_BIN) return false;
            o.ih = min((int)xf, AG_NEINT - 1);
        }
    }
    return true;
}

// FP32 directional factors (racc, rdon, Hramp) from the unit pair vector and
// the atom's staged bond vectors.  Returns false when cos_theta lies within
// its error bound of the D1/A2 branch at 0; the caller then uses pair_exact().
__device__ __forceinline__ bool angular_fast(int meta, float4 rvA, float4 rvB, int ia, float dX, float dY, float dZ,
                                             float rs, int ch, float3 rvh, PairQ<float> &o)
{
    o.racc = 1.f; o.rdon = 1.f; o.Hramp = 1.f;
    const bool dis = (meta & META_DIS) != 0;
    const int hb = (meta >> META_HB_SHIFT) & 7;
    if (hb != 2 && hb != 4 && hb != 5) return true;
    const float dn0 = dX * rs, dn1 = dY * rs, dn2 = dZ * rs;
    const float rv0 = rvA.x, rv1 = rvA.y, rv2 = rvA.z;
    const float cos_theta = ((0.f - dn0 * rv0) - dn1 * rv1) - dn2 * rv2;
    // An atom without bonded neighbours keeps a zero bond vector; its cos_theta
    // is exactly 0 in every precision, so the branch at 0 is not ambiguous.
    const bool rv_zero = (meta & META_RVZERO) != 0;
    if (hb == 2) {
        if (fabsf(cos_theta) < GUARD_COS && !rv_zero) return false;
        if (cos_theta <= 0.f) {
            o.racc = 0.f;
        } else {
            const int e = (meta >> META_REXP_SHIFT) & 7;
            o.racc = (e == 2) ? cos_theta * cos_theta
                   : (e == 4) ? (cos_theta * cos_theta) * (cos_theta * cos_theta) : cos_theta;
            if (ia != ch && ch >= 0) {
                float ct = rvh.x * rv0 + rvh.y * rv1 + rvh.z * rv2;
                ct = fminf(fmaxf(ct, -1.f), 1.f);
                // 0.5 - 0.5 cos(x) = 0.5 + 0.5 cos(x - pi), x - pi in [-pi, pi/3]: the
                // range on which __cosf's absolute error is within 2^-21.4
                o.Hramp = 0.5f + 0.5f * __cosf(acosf(ct) * (120.f / 90.f) - 3.14159265f);
            }
        }
    } else if (hb == 4) {
        o.rdon = (cos_theta <= 0.f) ? 0.f : cos_theta * cos_theta;
    } else if (!dis) {  // A2 ordered (main.cpp:3163-3246)
        if (fabsf(cos_theta) < GUARD_COS && !rv_zero) return false;
        const float w0 = rvB.x, w1 = rvB.y, w2 = rvB.z;
        float t0 = dn0 * w0 + dn1 * w1 + dn2 * w2;
        t0 = fminf(fmaxf(t0, -1.f), 1.f);
        // cos(pi/2 - acos(t0)) = sqrt(1 - t0^2)
        const float cos_t0 = sqrt_approx(fmaxf(1.f - t0 * t0, 0.f));
        const float c0 = dn1 * w2 - dn2 * w1, c1 = dn2 * w0 - dn0 * w2, c2 = dn0 * w1 - dn1 * w0;
        float rd2 = c0 * c0 + c1 * c1 + c2 * c2;
        rd2 = fmaxf(rd2, 1.0e-6f);
        const float inv_rd = rsqrtf(rd2);
        float ti = (c0 * rv0 + c1 * rv1 + c2 * rv2) * inv_rd;
        o.rdon = 0.f;
        if (cos_theta >= 0.f) {
            ti = fminf(fmaxf(ti, -1.f), 1.f);
            // sin(2|acos(ti) - pi/2|) = |sin(2 acos(ti))| = 2|ti|sqrt(1 - ti^2)
            const float s2 = 2.f * fabsf(ti) * sqrt_approx(fmaxf(1.f - ti * ti, 0.f));
            o.rdon = (0.9f + 0.1f * s2) * cos_t0;
        } else if (cos_theta >= -0.34202f) {
            const float b = 0.116978f - cos_theta * cos_theta;
            o.rdon = 562.25f * (b * b * b) * cos_t0;
        }
    } else {  // A2 disordered, cylindrical hydroxyl (main.cpp:3247-3272)
        const float ct = fminf(fmaxf(cos_theta, -1.f), 1.f);
        o.racc = 0.f; o.rdon = 0.f;
        // theta = acos(ct) <= 1.24791 + pi/2  <=>  ct >= -sin(1.24791); the value is 0 at the edge
        if (ct >= -0.94832352f) {
            // cos(theta - a) = ct cos(a) + sin(theta) sin(a), a = 1.24791
            const float c = ct * 0.31730505f + sqrtf(fmaxf(1.f - ct * ct, 0.f)) * 0.94832352f;
            o.rdon = (c * c) * (c * c);
            o.racc = o.rdon;
        }
    }
    return true;
}

// Exact distance of the reference's closest-H search (main.cpp:2994-3002).
__device__ __forceinline__ double h_dist(const DevProblem &p, int a, double cx, double cy, double cz)
{
    const double d0 = __dsub_rn(p.x[a], cx), d1 = __dsub_rn(p.y[a], cy), d2 = __dsub_rn(p.z[a], cz);
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
}

// ----------------------------------------------------------------- near ---
// One thread per grid point; bricks of 8x8x4 points inside one far-field frame.
//  stage  candidate atoms of the cells within 8.05 A of the brick, with their
//         canonical frame-relative FP32 coordinates and packed metadata,
//         ordered by receptor type (cell order within a type)
//  A      closest DS/D1 atom per point among the candidates (any DS/D1 atom
//         within 8.05 A of the point is a candidate, so a best distance
//         <= 8 A is the global minimum); FP32 prefilter, then FP64 with the
//         reference's order (strict '<' in file order == lowest index on a tie);
//         points with no DS/D1 atom within 8 A scan all of them (rare)
//  B      pair terms of every candidate inside 8 A (+ e-map near pairs)
// Per-point map accumulators.  The FP32 kernels keep them as pairs, so that
// a 16-byte table row (4 maps) adds as two packed adds; every add is the same
// IEEE addition as a scalar one, so the sums are unchanged.  Indices are
// compile-time constants wherever the kernels use them (unrolled loops), so
// the accumulators stay in registers.
template <class R, int NGK>
struct MapAcc {
    R v[NGK];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int m = 0; m < NGK; m++) v[m] = (R)0;
    }
    __device__ __forceinline__ R get(int m) const { return v[m]; }
    __device__ __forceinline__ void add(int m, R x) { v[m] += x; }
    __device__ __forceinline__ void add4(int m4, float4 T)
    {
        v[4 * m4] += (R)T.x; v[4 * m4 + 1] += (R)T.y;
        v[4 * m4 + 2] += (R)T.z; v[4 * m4 + 3] += (R)T.w;
    }
};
template <int NGK>
struct MapAcc<float, NGK> {
    float2 v[NGK / 2];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < NGK / 2; k++) v[k] = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ float get(int m) const { return (m & 1) ? v[m >> 1].y : v[m >> 1].x; }
    __device__ __forceinline__ void add(int m, float x)
    {
        if (m & 1) v[m >> 1].y += x;
        else v[m >> 1].x += x;
    }
    __device__ __forceinline__ void add4(int m4, float4 T)
    {
        v[2 * m4] = __fadd2_rn(v[2 * m4], make_float2(T.x, T.y));
        v[2 * m4 + 1] = __fadd2_rn(v[2 * m4 + 1], make_float2(T.z, T.w));
    }
};

// Accumulators a launch holds per point: groups of at most 8 maps (the
// 8-map sets of batched ensembles, config 0) run with 8, which frees 8 of
// the 80 registers; larger groups with NG_MAX.
constexpr int NGK_SMALL = 8;

// One brick `b` of one instance (p, g).
template <bool EXACT, int BX, int BY, int BZ, int NGK>
__device__ __forceinline__ void near_unit(const DevProblem &p, const NearGroup &g, const NearPtrs &ptr, int b,
                                          NearSmem &S)
{
    static_assert(BX * BY * BZ == NB_THREADS, "one thread per brick point");
    static_assert(FRAME_X % BX == 0 && FRAME_Y % BY == 0 && FRAME_Z % BZ == 0, "bricks tile far frames");
    using R = typename std::conditional<EXACT, double, float>::type;
    const int tid = threadIdx.x;
    for (int i = tid; i < NT_SMALL; i += NB_THREADS) {
        S.etab[i] = ptr.etab[i];
        S.sol[i] = ptr.solf[i];
    }
    __syncthreads();
    const int nbx = (p.n1x + BX - 1) / BX, nby = (p.n1y + BY - 1) / BY;
    const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
    // the brick's points inside the box, packed into its first wx*wy*wz threads
    // (x fastest), so that a brick on the box's edge leaves whole warps idle
    // instead of idle lanes in every warp; interior bricks: tid = x + BX*(y + BY*z)
    const int wx = min(BX, p.n1x - bx * BX), wy = min(BY, p.n1y - by * BY), wz = min(BZ, p.n1z - bz * BZ);
    const int ix = bx * BX + tid % wx, iy = by * BY + (tid / wx) % wy, iz = bz * BZ + tid / (wx * wy);
    const bool valid = tid < wx * wy * wz;
    const long long lin = ((long long)iz * p.n1y + iy) * p.n1x + ix;

    // far-kernel frame of this brick and the point's canonical coordinates
    const double sp128 = p.spacing * AG_A_DIV;
    const int ox = ((bx * BX) / FRAME_X) * FRAME_X, oy = ((by * BY) / FRAME_Y) * FRAME_Y,
              oz = ((bz * BZ) / FRAME_Z) * FRAME_Z;
    const double X0 = frame_origin_bins(ox, p.nex, sp128), Y0 = frame_origin_bins(oy, p.ney, sp128),
                 Z0 = frame_origin_bins(oz, p.nez, sp128);
    const float PX = frame_point_coord(ix - ox, sp128), PY = frame_point_coord(iy - oy, sp128),
                PZ = frame_point_coord(iz - oz, sp128);
    // FP64 point coordinates (main.cpp:2815-2859), formed where a pair needs them
    auto cx = [&]() { return (double)(ix - p.nex) * p.spacing; };
    auto cy = [&]() { return (double)(iy - p.ney) * p.spacing; };
    auto cz = [&]() { return (double)(iz - p.nez) * p.spacing; };

    const bool need_h = p.n_atom_maps > 0;
    const bool do_e = !EXACT && g.write_special && p.elec_map >= 0;
    const bool need_pairs = g.ng > 0 || (g.write_special && p.dsolv_map >= 0) || do_e;

    // candidate cells: brick bounding box grown by the candidate radius
    const double rc = AGB_NEAR_RADIUS;
    const double bx0 = (double)(bx * BX - p.nex) * p.spacing, bx1 = (double)(min(bx * BX + BX - 1, p.n1x - 1) - p.nex) * p.spacing;
    const double by0 = (double)(by * BY - p.ney) * p.spacing, by1 = (double)(min(by * BY + BY - 1, p.n1y - 1) - p.ney) * p.spacing;
    const double bz0 = (double)(bz * BZ - p.nez) * p.spacing, bz1 = (double)(min(bz * BZ + BZ - 1, p.n1z - 1) - p.nez) * p.spacing;
    auto cell_lo = [&](double v, double o, int n) { int c = (int)floor((v - rc - o) / p.cell_size); return max(0, min(n - 1, c)); };
    auto cell_hi = [&](double v, double o, int n) { int c = (int)floor((v + rc - o) / p.cell_size); return max(0, min(n - 1, c)); };
    const int cxl = cell_lo(bx0, p.cell0[0], p.ncx), cxh = cell_hi(bx1, p.cell0[0], p.ncx);
    const int cyl = cell_lo(by0, p.cell0[1], p.ncy), cyh = cell_hi(by1, p.cell0[1], p.ncy);
    const int czl = cell_lo(bz0, p.cell0[2], p.ncz), czh = cell_hi(bz1, p.cell0[2], p.ncz);
    const int nrow_y = cyh - cyl + 1;
    const int nseg_total = (need_pairs || need_h) ? nrow_y * (czh - czl + 1) : 0;

    // Stage chunk `c0` (nc candidates) of the laid-out segments, ordered by
    // receptor type by a stable counting sort (cell order within a type), so
    // that a warp's consecutive pairs read the table rows of one type, which
    // then stay in L1.  Slice k (candidates [32k, 32k + 32) of the chunk) is
    // ranked by one warp; S.tcnt[k][t] holds the slice's count of type t,
    // then the slot of its first such candidate.  All threads call it.
    static_assert(NB_CHUNK <= 2 * NB_THREADS && NB_CHUNK % 32 == 0, "two candidates per thread at most");
    auto stage = [&](int c0, int nc) {
        constexpr int NSL = NB_CHUNK / 32;
        for (int i = tid; i < NSL * 32; i += NB_THREADS) S.tcnt[i >> 5][i & 31] = 0;
        __syncthreads();
        int ca[2], ct[2], cr[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = u * NB_THREADS + tid;
            int a = -1, t = 32;  // lanes past the chunk form a group of their own
            if (i < nc) {
                const int c = c0 + i;
                int s = 0;
                while (S.seg_off[s + 1] <= c) s++;
                a = p.cell_atoms[S.seg_start[s] + (c - S.seg_off[s])];
                t = ptr.meta[a] & META_TYPE_MASK;
            }
            const unsigned same = __match_any_sync(0xffffffffu, t);
            cr[u] = __popc(same & ((1u << (tid & 31)) - 1u));
            if (i < nc && cr[u] == 0) S.tcnt[i >> 5][t] = __popc(same);
            ca[u] = a;
            ct[u] = t;
        }
        __syncthreads();
        if (tid < 32) {  // thread t: type t's slots, slices in order, after every lower type
            int run = 0;
            for (int k = 0; k < NSL; k++) {
                const int c = S.tcnt[k][tid];
                S.tcnt[k][tid] = run;
                run += c;
            }
            int incl = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += v;
            }
            for (int k = 0; k < NSL; k++) S.tcnt[k][tid] += incl - run;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int i = u * NB_THREADS + tid;
            if (i >= nc) continue;
            const int a = ca[u], j = S.tcnt[i >> 5][ct[u]] + cr[u];
            S.idx[j] = a;
            S.pos[j] = make_float4(frame_atom_coord(p.x[a] * AG_A_DIV, X0), frame_atom_coord(p.y[a] * AG_A_DIV, Y0),
                                   frame_atom_coord(p.z[a] * AG_A_DIV, Z0), (float)p.q[a]);
            S.a[j] = ptr.atomA[a];
            S.b[j] = ptr.atomB[a];
            const int m = ptr.meta[a];
            S.meta[j] = m;
            const int hb = (m >> META_HB_SHIFT) & 7;
            if (hb == 1 || hb == 2) S.hl[atomicAdd(&S.nh, 1)] = j;
        }
    };
    auto layout_segments = [&](int sb, int nseg) {
        if (tid == 0) {
            int off = 0;
            for (int s = 0; s < nseg; s++) {
                const int k = sb + s;
                const int cyy = cyl + k % nrow_y, czz = czl + k / nrow_y;
                const int c0 = (czz * p.ncy + cyy) * p.ncx + cxl, c1 = (czz * p.ncy + cyy) * p.ncx + cxh;
                const int st = p.cell_start[c0], en = p.cell_start[c1 + 1];
                S.seg_start[s] = st;
                S.seg_off[s] = off;
                off += en - st;
            }
            S.seg_off[nseg] = off;
            S.total = off;
            S.nh = 0;
        }
    };
    // the candidate list fits one chunk in the common case: stage it once
    bool resident = false;
    if (nseg_total > 0 && nseg_total <= NB_SEGS) {
        __syncthreads();
        layout_segments(0, nseg_total);
        __syncthreads();
        if (S.total <= NB_CHUNK) {
            stage(0, S.total);
            resident = true;
        }
        __syncthreads();
    }
    // visit every candidate chunk: fn(nc) with the chunk staged in shared memory.
    // One call site for fn, so its body is instantiated once.
    auto for_each_chunk = [&](auto &&fn) {
        const int nsb = resident ? 1 : (nseg_total + NB_SEGS - 1) / NB_SEGS;
        for (int sbi = 0; sbi < nsb; sbi++) {
            int total = S.total;
            if (!resident) {
                const int sb = sbi * NB_SEGS;
                __syncthreads();
                layout_segments(sb, min(NB_SEGS, nseg_total - sb));
                __syncthreads();
                total = S.total;
            }
            for (int c0 = 0; c0 < total; c0 += NB_CHUNK) {
                const int nc = min(NB_CHUNK, total - c0);
                if (!resident) {
                    __syncthreads();
                    if (tid == 0) S.nh = 0;
                    __syncthreads();
                    stage(c0, nc);
                    __syncthreads();
                }
                fn(nc);
            }
        }
    };
    // ---- A: closest DS/D1 hydrogen (main.cpp:2986-3015)
    int ch = -1;
    if (need_h) {
        // FP32 prefilter: the two smallest squared distances (bins^2) and the
        // atom of the smallest.  Every candidate within `lim` of the smallest
        // is re-checked in FP64; when the second smallest lies beyond `lim`,
        // that is the smallest's atom alone, and the FP64 pass over the
        // candidates reduces to its own distance.
        float best2 = 3.0e38f, next2 = 3.0e38f;
        int best_a = -1;
        for_each_chunk([&](int) {
            if (!valid) return;
            for (int k = 0; k < S.nh; k++) {
                const int j = S.hl[k];
                const float4 A = S.pos[j];
                const float dx = A.x - PX, dy = A.y - PY, dz = A.z - PZ;
                const float d2 = dx * dx + dy * dy + dz * dz;
                if (d2 < best2) {
                    next2 = best2;
                    best2 = d2;
                    best_a = S.idx[j];
                } else {
                    next2 = fminf(next2, d2);
                }
            }
        });
        const float lim = best2 * (1.0f + 2.0e-5f) + 4.0f;
        double rmin = 999999.;
        const bool several = valid && best_a >= 0 && next2 <= lim;
        if (valid && best_a >= 0 && !several) {
            rmin = h_dist(p, best_a, cx(), cy(), cz());
            ch = best_a;
        }
        if (__syncthreads_or(several))
            for_each_chunk([&](int) {
                if (!several) return;
                for (int k = 0; k < S.nh; k++) {
                    const int j = S.hl[k];
                    const float4 A = S.pos[j];
                    const float dx = A.x - PX, dy = A.y - PY, dz = A.z - PZ;
                    if (dx * dx + dy * dy + dz * dz > lim) continue;
                    const int a = S.idx[j];
                    const double r = h_dist(p, a, cx(), cy(), cz());
                    if (r < rmin || (r == rmin && a < ch)) { rmin = r; ch = a; }
                }
            });
        if (valid && !(rmin <= AG_NBC)) {  // nothing within 8 A: scan every DS/D1 atom in file order
            rmin = 999999.;
            ch = -1;
            for (int k = 0; k < p.n_h; k++) {
                const int a = p.h_index[k];
                const double r = h_dist(p, a, cx(), cy(), cz());
                if (r < rmin) { rmin = r; ch = a; }
            }
        }
    }
    float3 rvh = make_float3(0.f, 0.f, 0.f);
    if (!EXACT && ch >= 0) rvh = make_float3(ptr.atomA[ch].x, ptr.atomA[ch].y, ptr.atomA[ch].z);

    // ---- B: pair terms
    static_assert(NGK % 4 == 0 && NGK >= NG_MM && NGK <= NG_MAX, "accumulator count");
    MapAcc<R, NGK> E;
    R hmin[NG_MM], hmax[NG_MM];  // the FP64 twin only; FP32 keeps them in S
    E.zero();
#pragma unroll
    for (int m = 0; m < NG_MM; m++) {
        if (EXACT) { hmin[m] = 999999.; hmax[m] = -999999.; }
        else { S.hmin[m][tid] = 999999.f; S.hmax[m][tid] = -999999.f; }
    }
    uint32_t hflag = 0;
    R D1 = 0, D2 = 0, e_near = 0;
    unsigned n_near = 0, n_fb = 0;
    if (need_pairs) {
        // This warp's points as a box in frame bins (lanes outside the grid do
        // not count).  Per chunk, the warp keeps the staged atoms whose
        // distance to the box is within the near radius plus 2 bins, in staged
        // order: every pair a lane evaluates below (FP32 t < 1024 + GUARD_BIN,
        // or the FP64 twin's r^2 <= 64.0064) lies inside that margin, so the
        // pairs and their summation order are those of the full staged list.
        static_assert(NB_THREADS / 32 <= NB_WARPS_MAX, "per-warp candidate lists");
        const int lane = tid & 31, wid = tid >> 5;
        {
            float blo[3] = {valid ? PX : 3.0e38f, valid ? PY : 3.0e38f, valid ? PZ : 3.0e38f};
            float bhi[3] = {valid ? PX : -3.0e38f, valid ? PY : -3.0e38f, valid ? PZ : -3.0e38f};
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                    blo[d] = fminf(blo[d], __shfl_xor_sync(0xffffffffu, blo[d], o));
                    bhi[d] = fmaxf(bhi[d], __shfl_xor_sync(0xffffffffu, bhi[d], o));
                }
            if (lane == 0)
                for (int d = 0; d < 3; d++) {
                    S.wbox[wid][d] = blo[d];
                    S.wbox[wid][3 + d] = bhi[d];
                }
            __syncwarp();
        }
        const float keep2 = (FAR_T0 + 2.0f) * (FAR_T0 + 2.0f);
        unsigned short *wl = S.wl[wid];
        for_each_chunk([&](int nc) {
            int cnt = 0;
            for (int j0 = 0; j0 < nc; j0 += 32) {
                const int jj = j0 + lane;
                bool keep = false;
                if (jj < nc) {
                    const float4 A = S.pos[jj];
                    const float *bx = S.wbox[wid];
                    const float ex = fmaxf(fmaxf(bx[0] - A.x, A.x - bx[3]), 0.f);
                    const float ey = fmaxf(fmaxf(bx[1] - A.y, A.y - bx[4]), 0.f);
                    const float ez = fmaxf(fmaxf(bx[2] - A.z, A.z - bx[5]), 0.f);
                    keep = ex * ex + ey * ey + ez * ez <= keep2;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) wl[cnt + __popc(m & ((1u << lane) - 1u))] = (unsigned short)jj;
                cnt += __popc(m);
            }
            __syncwarp();
            if (!valid) return;
            for (int k = 0; k < cnt; k++) {
                const int j = wl[k];
                const int ia = S.idx[j];
                const int meta = S.meta[j];
                PairQ<R> q;
                bool e_pair = false;
                if (EXACT) {
                    const double d0 = __dsub_rn(p.x[ia], cx()), d1 = __dsub_rn(p.y[ia], cy()), d2 = __dsub_rn(p.z[ia], cz());
                    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
                    if (r2 > AG_NBC * AG_NBC * 1.0001) continue;
                    PairQ<double> qd;
                    pair_exact(p, ia, cx(), cy(), cz(), ch, qd);
                    if (!qd.ad4_in) continue;
                    q.ad4_in = 1; q.bin = qd.bin; q.bin_e = qd.bin_e; q.ih = qd.ih;
                    q.r = (R)qd.r; q.inv_rmax = (R)qd.inv_rmax; q.racc = (R)qd.racc; q.rdon = (R)qd.rdon; q.Hramp = (R)qd.Hramp;
                } else {
                    const float4 A = S.pos[j];
                    const float dY = __fsub_rn(A.y, PY), dZ = __fsub_rn(A.z, PZ);
                    const float s = __fmaf_rn(dY, dY, __fmaf_rn(dZ, dZ, TINY_T2));
                    const float dX = __fsub_rn(A.x, PX);
                    const float t2 = __fmaf_rn(dX, dX, s);
                    const float rs = rsqrt_approx(t2);
                    const float t = __fmul_rn(t2, rs);
                    if (t >= FAR_T0 + GUARD_BIN) continue;
                    e_pair = t < FAR_T0;  // the far-field kernel skips exactly these pairs
                    PairQ<float> qf;
                    if (!dist_fast(meta, t, rs, qf)) {
                        // through a copy: qf itself must not have its address
                        // taken, or it lives in local memory on the common path too
                        PairQ<float> qx = qf;
                        dist_exact_f(p, ia, cx(), cy(), cz(), qx);
                        qf = qx;
                        n_fb++;
                    }
                    qf.racc = 1.f; qf.rdon = 1.f; qf.Hramp = 1.f;
                    if (qf.ad4_in && !angular_fast(meta, S.a[j], S.b[j], ia, dX, dY, dZ, rs, ch, rvh, qf)) {
                        PairQ<double> qd;
                        pair_exact(p, ia, cx(), cy(), cz(), ch, qd);
                        qf.ad4_in = qd.ad4_in; qf.bin = qd.bin; qf.bin_e = qd.bin_e; qf.ih = qd.ih;
                        qf.r = (float)qd.r; qf.inv_rmax = (float)qd.inv_rmax; qf.racc = (float)qd.racc;
                        qf.rdon = (float)qd.rdon; qf.Hramp = (float)qd.Hramp;
                        n_fb++;
                    }
                    q.ad4_in = qf.ad4_in; q.bin = qf.bin; q.bin_e = qf.bin_e; q.ih = qf.ih;
                    q.r = qf.r; q.inv_rmax = qf.inv_rmax; q.racc = qf.racc; q.rdon = qf.rdon; q.Hramp = qf.Hramp;
                    if (e_pair && do_e) e_near += (R)(S.etab[min(q.bin_e, NT_SMALL - 1)] * A.w) * q.inv_rmax;
                    if (!q.ad4_in) continue;
                }
                n_near++;
                const int kr = min(q.bin, NT_SMALL - 1);
                const R sol = EXACT ? (R)p.sol_fn[kr] : (R)S.sol[kr];
                if (EXACT) {
                    D1 += (R)p.vol[ia] * sol;
                    D2 += (R)(p.solpar[ia] + p.solpar_q * fabs(p.q[ia])) * sol;
                } else {
                    D1 += (R)S.a[j].w * sol;  // vol
                    D2 += (R)S.b[j].w * sol;  // solpar + qasp|q|
                }
                if (g.ng == 0) continue;
                const int hb = (meta >> META_HB_SHIFT) & 7;
                const bool dis = (meta & META_DIS) != 0;
                const int ta = meta & META_TYPE_MASK;
                const int kn = min(q.bin, AG_NEINT - 1);
                const float4 *Trow = (const float4 *)(ptr.vdwT + ((size_t)ta * AG_NEINT + kn) * ptr.mpad + g.col0);
                const float4 *Hrow = (g.has_hrow && dis && p.hydrogen_type >= 0)
                    ? (const float4 *)(ptr.vdwT + ((size_t)p.hydrogen_type * AG_NEINT + q.ih) * ptr.mpad + g.col0) : Trow;
                if ((g.plain_hb >> hb) & 1u) {  // every map a plain sum for this class (most atoms)
#pragma unroll
                    for (int m4 = 0; m4 < NGK / 4; m4++) {
                        if (4 * m4 >= g.ng) break;
                        const float4 T4 = __ldg(Trow + m4);
                        E.add4(m4, T4);
                    }
                    continue;
                }
                const unsigned long long aw = g.actw[hb];
                const unsigned rows_plain = g.plain4 >> (4 * hb);
#pragma unroll
                for (int m4 = 0; m4 < NGK / 4; m4++) {
                    if (4 * m4 >= g.ng) break;
                    const float4 T4 = __ldg(Trow + m4);
                    if ((rows_plain >> m4) & 1u) {  // the same adds as the per-map chain below
                        E.add4(m4, T4);
                        continue;
                    }
                    float4 H4 = T4;
                    if (dis) H4 = __ldg(Hrow + m4);
                    const float Tv[4] = {T4.x, T4.y, T4.z, T4.w};
                    const float Hv[4] = {H4.x, H4.y, H4.z, H4.w};
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const int m = 4 * m4 + u;
                        const int act = (int)((aw >> (3 * m)) & 7ull);
                        if (act == ACT_SKIP) continue;
                        const R T = (R)Tv[u];
                        if (act == ACT_PLAIN) { E.add(m, T); continue; }
                        // FP32: a product with 0.01f (within 1.5 ulp of the quotient)
                        R rsph = EXACT ? T / (R)100. : T * (R)0.01f;
                        rsph = rsph > (R)0 ? rsph : (R)0;
                        rsph = rsph < (R)1 ? rsph : (R)1;
                        if (act == ACT_SUMA) {
                            const R Tv2 = dis ? (R)Hv[u] : T;
                            E.add(m, Tv2 * q.Hramp * (q.racc + ((R)1 - q.racc) * rsph));
                        } else if (act == ACT_MMD && dis) {
                            E.add(m, (R)Hv[u] * q.Hramp * (q.rdon + ((R)1 - q.rdon) * rsph));
                        } else if (m < NG_MM) {  // min/max maps are placed first by the host
                            const R f = (act == ACT_MMA) ? q.racc : q.rdon;
                            const R v = T * (f + ((R)1 - f) * rsph);
                            if (EXACT) {
                                hmin[m] = hmin[m] < v ? hmin[m] : v;
                                hmax[m] = hmax[m] > v ? hmax[m] : v;
                            } else {
                                const float a0 = S.hmin[m][tid], a1 = S.hmax[m][tid];
                                S.hmin[m][tid] = a0 < (float)v ? a0 : (float)v;
                                S.hmax[m][tid] = a1 > (float)v ? a1 : (float)v;
                            }
                            hflag |= 1u << m;
                        }
                    }
                }
            }
        });
    }

    // finalise (main.cpp:3420-3431) and store
    if (valid) {
#pragma unroll
        for (int m = 0; m < NGK; m++) {
            if (m >= g.ng) break;
            R v = E.get(m);
            if (m < NG_MM && (hflag & (1u << m))) {
                const R lo = EXACT ? hmin[m] : (R)S.hmin[m][tid], hi = EXACT ? hmax[m] : (R)S.hmax[m][tid];
                v += lo + (hi > (R)0 ? hi : (R)0);
            }
            v += (R)g.sp[m] * D1 + (R)g.vp[m] * D2;
            const size_t o = (size_t)g.out_map[m] * (size_t)p.P + (size_t)lin;
            if (g.cov[m]) {
                if (EXACT) ptr.out64[o] = ptr.cov_map[lin]; else ptr.out32[o] = (float)ptr.cov_map[lin];
            } else {
                if (EXACT) ptr.out64[o] = (double)v; else ptr.out32[o] = (float)v;
            }
        }
        if (g.write_special) {
            if (p.dsolv_map >= 0) {
                const size_t o = (size_t)p.dsolv_map * (size_t)p.P + (size_t)lin;
                const R d = (R)p.solpar_q * D1;
                if (EXACT) ptr.out64[o] = (double)d; else ptr.out32[o] = (float)d;
            }
            if (do_e)  // the near part of the e map; k_emap_reduce adds the far-field chunks
                ptr.out32[(size_t)p.elec_map * (size_t)p.P + (size_t)lin] = (float)e_near;
        }
    }
    if (ptr.counters) {  // one atomic per counter and warp
        const unsigned c0 = __reduce_add_sync(0xffffffffu, n_near), c1 = __reduce_add_sync(0xffffffffu, n_fb);
        if ((tid & 31) == 0) {
            if (c0) atomicAdd(ptr.counters + 0, (unsigned long long)c0);
            if (c1) atomicAdd(ptr.counters + 1, (unsigned long long)c1);
        }
    }
}

// Single instance: one CTA per brick.
template <bool EXACT, int BX, int BY, int BZ, int NGK>
__global__ void __launch_bounds__(NB_THREADS, NEAR_MIN_CTAS) k_near(DevProblem p, NearGroup g, NearPtrs ptr,
                                                                  int brick0)
{
    // The problem is read through a shared-memory copy: the FP64 fallbacks
    // take it by reference, and a reference to the kernel parameter would make
    // every thread copy it into local memory.
    __shared__ NearSmem S;
    __shared__ DevProblem s_p;
    if (threadIdx.x == 0) s_p = p;
    __syncthreads();
    near_unit<EXACT, BX, BY, BZ, NGK>(s_p, g, ptr, brick0 + blockIdx.x, S);
}

// Many instances, persistent: (instance-group, brick) units from an atomic
// counter; units never wait on each other.
template <int BX, int BY, int BZ, int NGK>
__global__ void __launch_bounds__(NB_THREADS, NEAR_MIN_CTAS)
k_near_batch(const NearInst *__restrict__ insts, const long long *__restrict__ unit_begin, int n_inst,
             unsigned long long *__restrict__ counter)
{
    __shared__ NearSmem S;
    __shared__ NearInst s_i;
    __shared__ long long s_unit;
    int cur = -1;
    const long long total = unit_begin[n_inst];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_unit = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long u = s_unit;
        if (u >= total) break;
        int lo = 0, hi = n_inst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (unit_begin[mid] <= u) lo = mid; else hi = mid - 1;
        }
        if (lo != cur) {
            __syncthreads();
            for (int i = threadIdx.x; i < (int)(sizeof(NearInst) / 4); i += NB_THREADS)
                ((int *)&s_i)[i] = ((const int *)&insts[lo])[i];
            __syncthreads();
            cur = lo;
        }
        near_unit<false, BX, BY, BZ, NGK>(s_i.p, s_i.g, s_i.ptr, (int)(u - unit_begin[lo]), S);
    }
}

// Covalent map(s), main.cpp:2866-2879, in FP64 (a handful of flops per point).
__global__ void k_covalent(DevProblem p, double *__restrict__ cov)
{
    const long long lin = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (lin >= p.P) return;
    const int ix = (int)(lin % p.n1x), iy = (int)((lin / p.n1x) % p.n1y), iz = (int)(lin / ((long long)p.n1x * p.n1y));
    const double d0 = __dsub_rn(p.cov_pos[0], (double)(ix - p.nex) * p.spacing);
    const double d1 = __dsub_rn(p.cov_pos[1], (double)(iy - p.ney) * p.spacing);
    const double d2 = __dsub_rn(p.cov_pos[2], (double)(iz - p.nez) * p.spacing);
    double rcov = __ddiv_rn(__dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2))),
                            p.cov_half_width);
    if (rcov < APPROX_ZERO_D) rcov = APPROX_ZERO_D;
    cov[lin] = __dmul_rn(p.cov_barrier, __dsub_rn(1., exp(__dmul_rn(__dmul_rn(log(0.5), rcov), rcov))));
}

}  // namespace agb

namespace agb {

int near_bricks(const DevProblem &p, int shape)
{
    int bx = 8, by = 8, bz = 4;
    if (shape == 1) { by = 4; bz = 8; }
    else if (shape == 2) { bx = 4; bz = 8; }
    return ((p.n1x + bx - 1) / bx) * ((p.n1y + by - 1) / by) * ((p.n1z + bz - 1) / bz);
}

cudaError_t launch_covalent(const DevProblem &p, double *cov, cudaStream_t s)
{
    k_covalent<<<(unsigned)((p.P + 255) / 256), 256, 0, s>>>(p, cov);
    return cudaGetLastError();
}

// Brick z-rows [bz0, bz1) (bz1 < 0: through the last).
cudaError_t launch_near(bool exact, const DevProblem &p, const NearGroup &g, const NearPtrs &ptr, int shape,
                        cudaStream_t s, int bz0, int bz1)
{
    int bx = 8, by = 8, bz = 4;
    if (!exact && shape == 1) { by = 4; bz = 8; }
    else if (!exact && shape == 2) { bx = 4; bz = 8; }
    const int nbx = (p.n1x + bx - 1) / bx, nby = (p.n1y + by - 1) / by, nbz = (p.n1z + bz - 1) / bz;
    if (bz1 < 0 || bz1 > nbz) bz1 = nbz;
    if (bz0 >= bz1) return cudaSuccess;
    const unsigned nb = (unsigned)(nbx * nby * (bz1 - bz0));
    const int b0 = bz0 * nbx * nby;
    const bool small = g.ng <= NGK_SMALL;
    if (exact) {
        k_near<true, 8, 8, 4, NG_MAX><<<nb, NB_THREADS, 0, s>>>(p, g, ptr, b0);
    } else if (shape == 1) {
        if (small) k_near<false, 8, 4, 8, NGK_SMALL><<<nb, NB_THREADS, 0, s>>>(p, g, ptr, b0);
        else k_near<false, 8, 4, 8, NG_MAX><<<nb, NB_THREADS, 0, s>>>(p, g, ptr, b0);
    } else if (shape == 2) {
        if (small) k_near<false, 4, 8, 8, NGK_SMALL><<<nb, NB_THREADS, 0, s>>>(p, g, ptr, b0);
        else k_near<false, 4, 8, 8, NG_MAX><<<nb, NB_THREADS, 0, s>>>(p, g, ptr, b0);
    } else {
        if (small) k_near<false, 8, 8, 4, NGK_SMALL><<<nb, NB_THREADS, 0, s>>>(p, g, ptr, b0);
        else k_near<false, 8, 8, 4, NG_MAX><<<nb, NB_THREADS, 0, s>>>(p, g, ptr, b0);
    }
    return cudaGetLastError();
}

template <int BX, int BY, int BZ, int NGK>
static cudaError_t near_batch_t(const NearInst *insts, const long long *unit_begin, int n_inst,
                                unsigned long long *counter, int ctas_per_sm, cudaStream_t s)
{
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_near_batch<BX, BY, BZ, NGK>, NB_THREADS, 0);
    const int per_sm = std::max(1, std::min(ctas_per_sm, occ));
    k_near_batch<BX, BY, BZ, NGK><<<sms * per_sm, NB_THREADS, 0, s>>>(insts, unit_begin, n_inst, counter);
    return cudaGetLastError();
}

template <int NGK>
static cudaError_t near_batch_shape(const NearInst *insts, const long long *unit_begin, int n_inst,
                                    unsigned long long *counter, int shape, int ctas_per_sm, cudaStream_t s)
{
    if (shape == 1) return near_batch_t<8, 4, 8, NGK>(insts, unit_begin, n_inst, counter, ctas_per_sm, s);
    if (shape == 2) return near_batch_t<4, 8, 8, NGK>(insts, unit_begin, n_inst, counter, ctas_per_sm, s);
    return near_batch_t<8, 8, 4, NGK>(insts, unit_begin, n_inst, counter, ctas_per_sm, s);
}

cudaError_t launch_near_batch(const NearInst *insts, const long long *unit_begin, int n_inst,
                              unsigned long long *counter, int shape, int ctas_per_sm, int max_ng, cudaStream_t s)
{
    if (max_ng <= NGK_SMALL)
        return near_batch_shape<NGK_SMALL>(insts, unit_begin, n_inst, counter, shape, ctas_per_sm, s);
    return near_batch_shape<NG_MAX>(insts, unit_begin, n_inst, counter, shape, ctas_per_sm, s);
}

}  // namespace agb
