// Per-pair arithmetic of the differentiable mode (kernels/diff.h states the
// mode): directional factors of main.cpp:3075-3272 with their partial
// derivatives, and the chain rule from the factors back to the pair vector and
// the bond vectors.  Written once for FP32 and FP64, host and device.
#pragma once
#include <cmath>

#include "diff.h"

#define DF_HD __host__ __device__ __forceinline__

namespace agb {
namespace dfm {

DF_HD float sqrt_(float v) { return sqrtf(v); }
DF_HD double sqrt_(double v) { return sqrt(v); }
DF_HD float acos_(float v) { return acosf(v); }
DF_HD double acos_(double v) { return acos(v); }
DF_HD float cos_(float v) { return cosf(v); }
DF_HD double cos_(double v) { return cos(v); }
DF_HD float sin_(float v) { return sinf(v); }
DF_HD double sin_(double v) { return sin(v); }
DF_HD float exp_(float v) { return expf(v); }
DF_HD double exp_(double v) { return exp(v); }
// cos and sin of x = 4 theta / 3, theta in [0, pi] (the Hramp angle).  FP32
// on the device through the shifted argument x - pi in [-pi, pi/3], on which
// __cosf and __sinf keep an absolute error within 2^-21.4.
DF_HD float cos43(float x)
{
#ifdef __CUDA_ARCH__
    return -__cosf(x - 3.14159265f);
#else
    return cosf(x);
#endif
}
DF_HD double cos43(double x) { return cos(x); }
DF_HD float sin43(float x)
{
#ifdef __CUDA_ARCH__
    return -__sinf(x - 3.14159265f);
#else
    return sinf(x);
#endif
}
DF_HD double sin43(double x) { return sin(x); }
// Square root, reciprocal square root and quotient inside the directional
// factors, which are continuous where these are used.  FP32 on the device:
// the hardware approximations (sqrt.approx, rsqrt.approx: a few ulp;
// __fdividef: 2 ulp for the divisors here, all above 1e-6); elsewhere the
// correctly rounded operations.
DF_HD float asqrt(float v)
{
#ifdef __CUDA_ARCH__
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(v));
    return y;
#else
    return sqrtf(v);
#endif
}
DF_HD double asqrt(double v) { return sqrt(v); }
DF_HD float arsqrt(float v)
{
#ifdef __CUDA_ARCH__
    float y;
    asm("rsqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(v));
    return y;
#else
    return 1.0f / sqrtf(v);
#endif
}
DF_HD double arsqrt(double v) { return 1.0 / sqrt(v); }
DF_HD float adiv(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
DF_HD double adiv(double a, double b) { return a / b; }
template <class R> DF_HD R mn(R a, R b) { return a < b ? a : b; }
template <class R> DF_HD R mx(R a, R b) { return a > b ? a : b; }
template <class R> DF_HD R ab(R a) { return a < R(0) ? -a : a; }

// sin / cos of the disordered-hydroxyl angle 1.24791 (main.cpp:3263)
constexpr double A2D_SIN = 0.9483235234688568, A2D_COS = 0.31730505012623506;
constexpr double DF_TINY = 1.0e-6;

// Directional factors of one pair and the partials the adjoint needs.
template <class R> struct Ang {
    R racc, rdon, H;
    R dacc_c, ddon_c;    // d racc / d cos_theta, d rdon / d cos_theta
    R ddon_t0, ddon_ti;  // A2 ordered: d rdon / d (dn . rv2), d rdon / d ti
    R dH_ct;             // d Hramp / d (rv_closestH . rv)
    R cr[3], rdi, tin;   // A2 ordered: dn x rv2, 1/|dn x rv2|, (dn x rv2) . rv
    bool rd_clamped;
};

// hb: receptor hbond class; dis: disorder flag; ramp: Hramp applies (the
// point's closest DS/D1 atom exists and is not this atom).
// dn = (atom - point)/r; rvh = bond vector of the point's closest DS/D1 atom.
// The factors of a pair without directional terms: all 1, no partials.
template <class R>
DF_HD void ang_plain(Ang<R> &o)
{
    o.racc = R(1); o.rdon = R(1); o.H = R(1);
    o.dacc_c = R(0); o.ddon_c = R(0); o.ddon_t0 = R(0); o.ddon_ti = R(0); o.dH_ct = R(0);
    o.cr[0] = o.cr[1] = o.cr[2] = R(0); o.rdi = R(0); o.tin = R(0); o.rd_clamped = true;
}

template <class R>
DF_HD void angular(int hb, int rexp, bool dis, bool ramp, const R dn[3], const R rv[3], const R rv2[3],
                   const R rvh[3], Ang<R> &o)
{
    ang_plain(o);
    if (hb != 2 && hb != 4 && hb != 5) return;
    const R c = -(dn[0] * rv[0] + dn[1] * rv[1] + dn[2] * rv[2]);
    if (hb == 2) {  // D1 (main.cpp:3075-3132)
        if (c > R(0)) {
            if (rexp == 2) { o.racc = c * c; o.dacc_c = R(2) * c; }
            else if (rexp == 4) { const R c2 = c * c; o.racc = c2 * c2; o.dacc_c = R(4) * c2 * c; }
            else { o.racc = c; o.dacc_c = R(1); }
        } else {
            o.racc = R(0);
        }
        if (ramp) {  // evaluated for every D1 pair in this mode
            R ct = rvh[0] * rv[0] + rvh[1] * rv[1] + rvh[2] * rv[2];
            const bool inside = ct < R(1) && ct > R(-1);
            ct = mn(mx(ct, R(-1)), R(1));
            const R th = acos_(ct);
            o.H = R(0.5) - R(0.5) * cos43(th * R(4.0 / 3.0));
            if (inside) {
                const R s = asqrt(R(1) - ct * ct);
                o.dH_ct = (s > R(DF_TINY)) ? adiv(R(-2.0 / 3.0) * sin43(th * R(4.0 / 3.0)), s)
                                           : (ct > R(0) ? R(-8.0 / 9.0) : R(0));
            }
        }
    } else if (hb == 4) {  // A1 (main.cpp:3133-3162)
        if (c > R(0)) { o.rdon = c * c; o.ddon_c = R(2) * c; }
        else o.rdon = R(0);
    } else if (!dis) {  // A2 ordered (main.cpp:3163-3246)
        R t0 = dn[0] * rv2[0] + dn[1] * rv2[1] + dn[2] * rv2[2];
        const bool t0_in = t0 < R(1) && t0 > R(-1);
        t0 = mn(mx(t0, R(-1)), R(1));
        const R ct0 = asqrt(mx(R(1) - t0 * t0, R(0)));  // cos(pi/2 - acos(t0))
        const R dct0 = (t0_in && ct0 > R(DF_TINY)) ? adiv(-t0, ct0) : R(0);
        o.cr[0] = dn[1] * rv2[2] - dn[2] * rv2[1];
        o.cr[1] = dn[2] * rv2[0] - dn[0] * rv2[2];
        o.cr[2] = dn[0] * rv2[1] - dn[1] * rv2[0];
        R rd2 = o.cr[0] * o.cr[0] + o.cr[1] * o.cr[1] + o.cr[2] * o.cr[2];
        o.rd_clamped = rd2 < R(DF_TINY);
        rd2 = mx(rd2, R(DF_TINY));
        o.rdi = arsqrt(rd2);
        o.tin = o.cr[0] * rv[0] + o.cr[1] * rv[1] + o.cr[2] * rv[2];
        R ti = o.tin * o.rdi;
        const bool ti_in = ti < R(1) && ti > R(-1);
        ti = mn(mx(ti, R(-1)), R(1));
        const R sq = asqrt(mx(R(1) - ti * ti, R(0)));
        const R s2 = R(2) * ab(ti) * sq;  // sin(2 |acos(ti) - pi/2|)
        const R ds2 = (ti_in && sq > R(DF_TINY)) ? (ti >= R(0) ? R(2) : R(-2)) * adiv(R(1) - R(2) * ti * ti, sq) : R(0);
        if (c >= R(0)) {
            const R base = R(0.9) + R(0.1) * s2;
            o.rdon = base * ct0;
            o.ddon_t0 = base * dct0;
            o.ddon_ti = R(0.1) * ds2 * ct0;
        } else if (c >= R(-0.34202)) {
            const R bb = R(0.116978) - c * c;
            const R k = R(1) + adiv(s2, R(9));  // continuity factor of this mode
            const R p3 = R(562.25) * bb * bb * bb;
            o.rdon = p3 * ct0 * k;
            o.ddon_c = R(562.25) * R(3) * bb * bb * (R(-2) * c) * ct0 * k;
            o.ddon_t0 = p3 * k * dct0;
            o.ddon_ti = adiv(p3 * ct0 * ds2, R(9));
        } else {
            o.rdon = R(0);
        }
    } else {  // A2 disordered hydroxyl (main.cpp:3247-3272)
        const bool c_in = c < R(1) && c > R(-1);
        const R ct = mn(mx(c, R(-1)), R(1));
        o.racc = R(0); o.rdon = R(0);
        if (ct >= R(-A2D_SIN)) {
            const R sq = asqrt(mx(R(1) - ct * ct, R(0)));
            const R cc = ct * R(A2D_COS) + sq * R(A2D_SIN);  // cos(acos(ct) - 1.24791)
            const R c2 = cc * cc;
            o.rdon = o.racc = c2 * c2;
            const R dcc = (c_in && sq > R(DF_TINY)) ? R(A2D_COS) - adiv(ct * R(A2D_SIN), sq) : R(0);
            o.dacc_c = o.ddon_c = R(4) * c2 * cc * dcc;
        }
    }
}

// Chain rule from upstream gradients of (racc, rdon, Hramp) to the unit pair
// vector dn and the bond vectors (accumulated).
template <class R>
DF_HD void angular_bwd(int hb, bool dis, const Ang<R> &o, R G_racc, R G_rdon, R G_H, const R dn[3], const R rv[3],
                       const R rv2[3], const R rvh[3], R g_dn[3], R g_rv[3], R g_rv2[3], R g_rvh[3])
{
    if (hb != 2 && hb != 4 && hb != 5) return;
    const R g_c = G_racc * o.dacc_c + G_rdon * o.ddon_c;  // cos_theta = -dn . rv
    for (int i = 0; i < 3; i++) { g_dn[i] -= g_c * rv[i]; g_rv[i] -= g_c * dn[i]; }
    if (hb == 2) {
        const R g_ct = G_H * o.dH_ct;  // ct = rvh . rv
        for (int i = 0; i < 3; i++) { g_rv[i] += g_ct * rvh[i]; g_rvh[i] += g_ct * rv[i]; }
    } else if (hb == 5 && !dis) {
        const R g_t0 = G_rdon * o.ddon_t0;  // t0 = dn . rv2
        for (int i = 0; i < 3; i++) { g_dn[i] += g_t0 * rv2[i]; g_rv2[i] += g_t0 * dn[i]; }
        const R g_ti = G_rdon * o.ddon_ti;  // ti = (cr . rv) / |cr|
        const R g_tin = g_ti * o.rdi;
        const R g_rd = o.rd_clamped ? R(0) : -g_ti * o.tin * o.rdi * o.rdi * o.rdi;
        R g_cr[3];
        for (int i = 0; i < 3; i++) {
            g_rv[i] += g_tin * o.cr[i];
            g_cr[i] = g_tin * rv[i] + g_rd * o.cr[i];
        }
        // cr = dn x rv2
        g_dn[0] += rv2[1] * g_cr[2] - rv2[2] * g_cr[1];
        g_dn[1] += rv2[2] * g_cr[0] - rv2[0] * g_cr[2];
        g_dn[2] += rv2[0] * g_cr[1] - rv2[1] * g_cr[0];
        g_rv2[0] += g_cr[1] * dn[2] - g_cr[2] * dn[1];
        g_rv2[1] += g_cr[2] * dn[0] - g_cr[0] * dn[2];
        g_rv2[2] += g_cr[0] * dn[1] - g_cr[1] * dn[0];
    }
}

// Linear interpolation of a (value, step) table at bin b, fraction f.
template <class R> DF_HD R lerp(const R2<R> &e, R f) { return e.v + f * e.d; }

// rsph = clamp(T / 100, 0, 1) (main.cpp:3293-3296) and its derivative.
template <class R> DF_HD R rsph(R T, R &d)
{
    const R s = T * R(0.01);
    if (s <= R(0)) { d = R(0); return R(0); }
    if (s >= R(1)) { d = R(0); return R(1); }
    d = R(0.01);
    return s;
}


// One staged receptor atom.
template <class R> struct Atom {
    R x, y, z, q, vol, solpar, rv[3], rv2[3];
    int meta, idx;
};

// Geometry of one pair: d = atom - point, x = A_DIV r, switch w(x) and the
// desolvation factor sol(x).
template <class R> struct Geom {
    R d[3], dn[3], r, inv, x, fx, w, dw, sol, dsol;
    int b;
};

// r = max(|d|, DF_TINY) and 1 / r from r^2.  r is the correctly rounded
// square root everywhere (it picks the table bin, and the adjoint's slopes
// jump at bin edges); FP32 on the device takes 1 / r from one rsqrt.approx
// (about 2 ulp) instead of a division.
DF_HD void dist_inv(double r2, double &r, double &inv)
{
    r = sqrt(r2);
    if (r < DF_TINY) r = DF_TINY;
    inv = 1.0 / r;
}
DF_HD void dist_inv(float r2, float &r, float &inv)
{
#ifdef __CUDA_ARCH__
    r = sqrtf(r2);
    if (r < float(DF_TINY)) r = float(DF_TINY);
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(r * r));
#else
    r = sqrtf(r2);
    if (r < float(DF_TINY)) r = float(DF_TINY);
    inv = 1.0f / r;
#endif
}

// False when the pair adds nothing: beyond 8 A, or a disordered hydrogen that
// LOOP 2 skips (main.cpp:3052).  sol may be null when no slot reads the
// desolvation table (sol and dsol are then 0).
template <class R>
DF_HD bool geom(const R2<R> *sol, const Atom<R> &at, R px, R py, R pz, Geom<R> &g)
{
    if (at.meta & DM_SKIP) return false;
    g.d[0] = at.x - px; g.d[1] = at.y - py; g.d[2] = at.z - pz;
    const R r2 = g.d[0] * g.d[0] + g.d[1] * g.d[1] + g.d[2] * g.d[2];
    if (r2 > R(AG_NBC * AG_NBC)) return false;
    R r, inv;
    dist_inv(r2, r, inv);
    g.r = r;
    g.inv = inv;
    for (int i = 0; i < 3; i++) g.dn[i] = g.d[i] * inv;
    g.x = r * R(AG_A_DIV);
    int b = (int)g.x;
    b = b < AG_NEINT - 1 ? b : AG_NEINT - 1;
    g.b = b;
    g.fx = g.x - R(b);
    const R room = R(AG_NEINT) - g.x;
    g.w = room < R(1) ? room : R(1);
    g.dw = room < R(1) ? R(-1) : R(0);
    if (sol) {
        g.sol = lerp(sol[b], g.fx);
        g.dsol = sol[b].d;
    } else {
        g.sol = R(0);
        g.dsol = R(0);
    }
    return true;
}

// T_H(r - 1.10): the hydrogen row at xh = A_DIV (r - 1.10) (main.cpp:3309-3313).
template <class R>
DF_HD R th_lookup(const DiffArgs &a, const R2<R> *vdw, int s, R x, R &dth)
{
    dth = R(0);
    if (a.hydrogen_type < 0 || a.hydrogen_type >= a.n_rec_types) return R(0);
    const R2<R> *row = vdw + (size_t)a.hydrogen_type * AG_NEINT * a.tab_stride + s;
    const R xh = x - R(1.10 * AG_A_DIV);
    if (xh <= R(0)) return row[0].v;
    int bh = (int)xh;
    bh = bh < AG_NEINT - 1 ? bh : AG_NEINT - 1;
    const R2<R> e = row[(size_t)bh * a.tab_stride];
    dth = e.d;
    return lerp(e, xh - R(bh));
}

// The value v of an H-bond-aware pair term and its partials (main.cpp:3297-3375).
template <class R> struct Term {
    R v, dT, dTH, dracc, drdon, dH, dx;  // dx: total d v / d x through both tables
};

// te: the pair's table entry (value, slope) for slot s.
template <class R>
DF_HD void term(const DiffArgs &a, const R2<R> *vdw, int act, const R2<R> &te, int s, const Geom<R> &g,
                const Ang<R> &an, Term<R> &t)
{
    const R T = lerp(te, g.fx);
    R drs;
    const R rs = rsph(T, drs);
    t.dT = R(0); t.dTH = R(0); t.dracc = R(0); t.drdon = R(0); t.dH = R(0);
    R dth = R(0);
    switch (act) {
        case DA_PLAIN:
            t.v = T; t.dT = R(1);
            break;
        case DA_SUMA: {
            const R f = an.racc + (R(1) - an.racc) * rs;
            t.v = T * an.H * f;
            t.dT = an.H * f + T * an.H * (R(1) - an.racc) * drs;
            t.dracc = T * an.H * (R(1) - rs);
            t.dH = T * f;
        } break;
        case DA_SUMA_DIS: {
            const R TH = th_lookup(a, vdw, s, g.x, dth);
            const R f = an.racc + (R(1) - an.racc) * rs;
            t.v = TH * an.H * f;
            t.dTH = an.H * f;
            t.dT = TH * an.H * (R(1) - an.racc) * drs;
            t.dracc = TH * an.H * (R(1) - rs);
            t.dH = TH * f;
        } break;
        case DA_MMA: {
            const R f = an.racc + (R(1) - an.racc) * rs;
            t.v = T * f;
            t.dT = f + T * (R(1) - an.racc) * drs;
            t.dracc = T * (R(1) - rs);
        } break;
        case DA_SUMD_DIS: {
            const R TH = th_lookup(a, vdw, s, g.x, dth);
            const R f = an.rdon + (R(1) - an.rdon) * rs;
            t.v = TH * an.H * f;
            t.dTH = an.H * f;
            t.dT = TH * an.H * (R(1) - an.rdon) * drs;
            t.drdon = TH * an.H * (R(1) - rs);
            t.dH = TH * f;
        } break;
        case DA_MMD: {
            const R f = an.rdon + (R(1) - an.rdon) * rs;
            t.v = T * f;
            t.dT = f + T * (R(1) - an.rdon) * drs;
            t.drdon = T * (R(1) - rs);
        } break;
        default:
            t.v = R(0);
            break;
    }
    t.dx = t.dT * te.d + t.dTH * dth;
}

DF_HD bool act_is_mm(int act) { return act == DA_MMA || act == DA_MMD; }

// The first n (<= MS) entries of a table row.  FP32 on the device reads two
// slots per 16-byte load: rows hold tab_stride (a multiple of 4) entries of
// 8 bytes, so every row starts 16-byte aligned.
template <class R, int MS>
DF_HD void load_row(const R2<R> *row, int n, R2<R> *out)
{
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 4 && MS % 2 == 0) {
        const float4 *r4 = reinterpret_cast<const float4 *>(row);
#pragma unroll
        for (int k = 0; k < MS / 2; k++)
            if (2 * k < n) {
                const float4 v = __ldg(r4 + k);
                out[2 * k] = R2<R>{v.x, v.y};
                out[2 * k + 1] = R2<R>{v.z, v.w};
            }
        return;
    }
#endif
#pragma unroll
    for (int s = 0; s < MS; s++)
        if (s < n) out[s] = row[s];
}

// Forward: add one pair to the point's slot energies and min/max registers.
// MS, MM: the slots and min/max registers a kernel instantiation holds
// (at least a.n_slots and a.n_mm).
template <class R, int MS = DF_MAXS, int MM = DF_MAXMM>
DF_HD void pair_fwd(const DiffArgs &a, const R2<R> *vdw, const Geom<R> &g, const Atom<R> &at, const Ang<R> &an,
                    R *E, R *hmin, R *hmax, int *amin, int *amax)
{
    const int type = at.meta & DM_TYPE_MASK, hb = (at.meta >> DM_HB_SHIFT) & 7;
    const int cls = hb + ((at.meta & DM_DIS) ? 8 : 0);
    const R qasp = R(a.solpar_q);
    const R solv = at.solpar + qasp * ab(at.q);
    R2<R> te[MS];
    load_row<R, MS>(vdw + ((size_t)type * AG_NEINT + g.b) * a.tab_stride, a.n_slots, te);
#pragma unroll
    for (int s = 0; s < MS; s++) {
        if (s >= a.n_slots) break;
        const int kind = a.slot_kind[s];
        if (kind == DK_D) {  // main.cpp:3393-3404
            E[s] += g.w * qasp * at.vol * g.sol;
            continue;
        }
        const int m = a.slot_tab[s];
        if (m >= 0) {
            const int act = a.act[s][cls];
            if (act != DA_NONE) {
                Term<R> t;
                term(a, vdw, act, te[s], s, g, an, t);
                const R val = g.w * t.v;
                if (act_is_mm(act)) {
                    if (s < MM) {  // min/max slots come first
                        if (val <= hmin[s]) { hmin[s] = val; amin[s] = at.idx; }
                        if (val >= hmax[s]) { hmax[s] = val; amax[s] = at.idx; }
                    }
                } else {
                    E[s] += val;
                }
            }
        }
        if (a.slot_desolv[s])  // main.cpp:3381-3389
            E[s] += g.w * g.sol * (R(a.slot_sp[s]) * at.vol + R(a.slot_vp[s]) * solv);
    }
}

// Adjoint of pair_fwd for one pair: upstream gradients gs[] of the point's
// slots; amin/amax: the atoms that attain the point's min/max (amax < 0 when
// max(hmax, 0) = 0).  Returns d L / d x (x = A_DIV r), d L / d (racc, rdon,
// Hramp) and d L / d q.
template <class R, int MS = DF_MAXS, int MM = DF_MAXMM>
DF_HD void pair_bwd(const DiffArgs &a, const R2<R> *vdw, const Geom<R> &g, const Atom<R> &at, const Ang<R> &an,
                    const R *gs, const int *amin, const int *amax, R &G_x, R &G_racc, R &G_rdon, R &G_H, R &G_q)
{
    const int type = at.meta & DM_TYPE_MASK, hb = (at.meta >> DM_HB_SHIFT) & 7;
    const int cls = hb + ((at.meta & DM_DIS) ? 8 : 0);
    const R qasp = R(a.solpar_q);
    const R solv = at.solpar + qasp * ab(at.q);
    const R sgnq = at.q > R(0) ? R(1) : (at.q < R(0) ? R(-1) : R(0));
    const R dsol_x = g.dw * g.sol + g.w * g.dsol;  // d (w sol) / d x
    const R2<R> *row = vdw + ((size_t)type * AG_NEINT + g.b) * a.tab_stride;
    R2<R> tp[2];  // table entries of slots s & ~1 and (s & ~1) + 1
#pragma unroll
    for (int s = 0; s < MS; s++) {
        if (s >= a.n_slots) break;
        if ((s & 1) == 0) load_row<R, 2>(row + s, a.n_slots - s, tp);
        const int kind = a.slot_kind[s];
        const R gsl = gs[s];
        if (kind == DK_D) {
            G_x += gsl * qasp * at.vol * dsol_x;
            continue;
        }
        const int m = a.slot_tab[s];
        if (m >= 0) {
            const int act = a.act[s][cls];
            if (act != DA_NONE) {
                R gv = gsl;
                if (act_is_mm(act)) {
                    gv = R(0);
                    if (s < MM) {
                        if (amin[s] == at.idx) gv += gsl;
                        if (amax[s] == at.idx) gv += gsl;
                    }
                }
                if (gv != R(0)) {
                    Term<R> t;
                    term(a, vdw, act, tp[s & 1], s, g, an, t);
                    G_x += gv * (g.dw * t.v + g.w * t.dx);
                    G_racc += gv * g.w * t.dracc;
                    G_rdon += gv * g.w * t.drdon;
                    G_H += gv * g.w * t.dH;
                }
            }
        }
        if (a.slot_desolv[s]) {
            const R sp = R(a.slot_sp[s]), vp = R(a.slot_vp[s]);
            G_x += gsl * dsol_x * (sp * at.vol + vp * solv);
            G_q += gsl * g.w * g.sol * vp * qasp * sgnq;
        }
    }
}

// d L / d (atom position) of one pair from d L / d x and d L / d dn.
template <class R>
DF_HD void geom_bwd(const Geom<R> &g, R G_x, const R g_dn[3], R g_d[3])
{
    const R gr = G_x * R(AG_A_DIV);
    const R ddot = g.dn[0] * g_dn[0] + g.dn[1] * g_dn[1] + g.dn[2] * g_dn[2];
    for (int i = 0; i < 3; i++) g_d[i] = gr * g.dn[i] + (g_dn[i] - g.dn[i] * ddot) * g.inv;
}

}  // namespace dfm
}  // namespace agb
