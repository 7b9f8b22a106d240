// Electrostatic map kernels (replace LOOP 1 of the reference, main.cpp:2940-2982).
//
// k_emap_far  -- production FP32 far field: every (point, atom) pair whose
//                canonical FP32 distance t = A_DIV*r is >= AG_NEINT bins
//                (r >= 8 A).  Pairs nearer than that are left to the near-field
//                kernel, which evaluates them with exact bins.  Per pair:
//                1 rsqrt (MUFU), packed FP32x2 arithmetic, one shared-memory
//                table gather.  Atoms are streamed through shared memory in
//                tiles; each thread keeps 8 grid points of one x-row in
//                registers (two-level summation: per-tile partial + total).
//                The atom list is split into chunks for load balance; chunk
//                partial sums land in far_partial[chunk][point].
// k_emap_reduce -- the e map: chunk partials added in fixed chunk order, then
//                the near-field part the near kernel left in the map
//                (deterministic; lets the far and near kernels run
//                concurrently).
// k_emap_exact -- FP64 twin: every pair, exactly the reference expression
//                (nested hypot, double table), file order summation.
#include <algorithm>

#include "agb_device.cuh"
#include "kernels.h"

namespace agb {

constexpr int EF_THREADS = 256;
// float2 pairs of points per thread: 8 points of one x-row, FRAME_X wide
constexpr int EF_PAIRS = FRAME_X / 8;

__device__ __forceinline__ float lds_f32(uint32_t addr)
{
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}

constexpr int FAR_TIE_FLAG = 1 << 30;

// The instance's far table into shared memory: a.tab_len floats (a multiple
// of 4) of far_tab.
__device__ __forceinline__ void load_far_table(float4 *s_tab4, const FarArgs &a)
{
    for (int i = threadIdx.x; i < a.tab_len / 4; i += EF_THREADS) s_tab4[i] = __ldg(((const float4 *)a.far_tab) + i);
}

// Exact LOOP 1 bin of a far pair whose guard bins differ (kb and kb + 1):
// the reference's bin (int)(r*A_DIV) with r = hypot(dx, hypot(dy, dz))
// (main.cpp:97, :2951-2956).  The FP64 differences are the reference's
// coordinate differences scaled by A_DIV = 2^7 (exact: x*A_DIV, and the grid
// coordinate ((i - ne)*spacing)*A_DIV = (i - ne)*(spacing*A_DIV); ix, iy, iz
// are i - ne); the squared distance decides against the edge (kb + 1)^2
// unless it lies within 1e-12 of it, where the reference's own expression
// decides and the result carries FAR_TIE_FLAG.
__device__ __forceinline__ int far_exact_bin(const double *ax128, const double *ay128, const double *az128, int at,
                                             double spacing_adiv, int ix, int iy, int iz, int kb)
{
    const double dx = __dsub_rn(__ldg(ax128 + at), __dmul_rn((double)ix, spacing_adiv));
    const double dy = __dsub_rn(__ldg(ay128 + at), __dmul_rn((double)iy, spacing_adiv));
    const double dz = __dsub_rn(__ldg(az128 + at), __dmul_rn((double)iz, spacing_adiv));
    const double t2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    const double e = (double)(kb + 1), e2 = __dmul_rn(e, e);  // exact: kb < 2^23
    if (fabs(__dsub_rn(t2, e2)) > 1.0e-12 * e2) return t2 >= e2 ? kb + 1 : kb;
    const double inv = 1.0 / AG_A_DIV;  // exact
    const double r = hypot(__dmul_rn(dx, inv), hypot(__dmul_rn(dy, inv), __dmul_rn(dz, inv)));
    return (int)__dmul_rn(r, (double)AG_A_DIV) | FAR_TIE_FLAG;
}

// The guard bins of a packed pair of distances: bit patterns MAGIC_BITS +
// floor(t*edge_lo) and MAGIC_BITS + floor(t*edge_hi) (one FMA each, rounded
// toward zero onto 2^23).
__device__ __forceinline__ void far_guard_bins(float2 t, float2 lom, float2 him, float2 &lo, float2 &hi)
{
    const float2 magic = make_float2(8388608.f, 8388608.f);
    lo = __ffma2_rz(t, lom, magic);
    hi = __ffma2_rz(t, him, magic);
}

// A thread's place in a far-field unit: the compact 4x4x2 lane footprint per
// warp (fewest table bank conflicts); each thread holds 8 points of one
// x-row, x = tx + 8j and tx + 8j + 4 (j < EF_PAIRS).
struct FarLane {
    int tx, ty, tz;
    bool warp_in;  // some row and plane of the warp lie inside the box
};
__device__ __forceinline__ FarLane far_lane(const FarArgs &a, int tid, int oy, int oz)
{
    const int lane = tid & 31, w = tid >> 5;
    FarLane l;
    l.tx = lane & 3;
    l.ty = ((lane >> 2) & 3) + 4 * (w & 1);
    l.tz = (lane >> 4) + 2 * (w >> 1);
    l.warp_in = oy + 4 * (w & 1) < a.n1y && oz + 2 * (w >> 1) < a.n1z;
    return l;
}

// Edge-bit words of unit (f, chunk): a.edge_words words per thread, word k
// of thread tid at [(chunk * nframes + f) * edge_words + k] * EF_THREADS + tid.
__device__ __forceinline__ size_t far_bits_base(const FarArgs &a, int f, int chunk)
{
    return ((size_t)chunk * (size_t)(a.nfx * a.nfy * a.nfz) + (size_t)f) * (size_t)a.edge_words * EF_THREADS;
}

// One work unit: frame `f` of one instance against atom chunk `chunk`.
// The caller has loaded the instance's table into s_tab4 and synchronised.
// Atom tile entries: frame-relative (Y, Z, X) in bins and w = q*coeff_estat*A_DIV,
// in that order so that (Y, Z) arrive in an aligned register pair, the operand
// of the packed y/z difference: with (X, Y, Z, w) the pair needed moves, and
// the kernel took 8.20 against 7.89 ms for 127^3 points x 10,000 atoms.
// The first NJ pairs of each thread hold the frame's x columns inside the box
// (the rest is padding and is skipped), and a warp whose 4 rows or 2 planes
// all lie past the box skips the pairs.
//
// Table bins (FAR_TAB_TABLE).  Each pair's table value is T[floor(t*edge_lo)];
// a pair whose second guard bin floor(t*edge_hi) differs lies within the FP32
// error bound of a bin edge.  Each thread records one bit per atom with such
// a pair among its own, one 32-bit word per 32 atoms, in a.edge_bits; the
// fix-up kernel (k_far_fixup) resolves those pairs afterwards.
// CLAMP: t is clamped half a bin past the last bin; without it the table
// extends past bin NDIEL-1 (repeating that bin's value) to a length that
// covers every distance of the instance, which saves the per-pair clamp.
template <int TILE, int MODE, int NJ, bool CLAMP>
__device__ __forceinline__ void far_unit_n(const FarArgs &a, int f, int chunk, const float4 *s_tab4, float4 *s_atom)
{
    const int tid = threadIdx.x;
    const int fx = f % a.nfx, fy = (f / a.nfx) % a.nfy, fz = f / (a.nfx * a.nfy);
    const int ox = fx * FRAME_X, oy = fy * FRAME_Y, oz = fz * FRAME_Z;
    // frame origin in bins, exactly (ox-nex)*spacing*A_DIV as the reference forms c (main.cpp:2859)
    const double X0 = frame_origin_bins(ox, a.nex, a.spacing_adiv);
    const double Y0 = frame_origin_bins(oy, a.ney, a.spacing_adiv);
    const double Z0 = frame_origin_bins(oz, a.nez, a.spacing_adiv);
    const FarLane L = far_lane(a, tid, oy, oz);
    const float py = frame_point_coord(L.ty, a.spacing_adiv);
    const float pz = frame_point_coord(L.tz, a.spacing_adiv);
    float2 npx[NJ];
#pragma unroll
    for (int j = 0; j < NJ; j++)
        npx[j] = make_float2(-frame_point_coord(L.tx + 8 * j, a.spacing_adiv),
                             -frame_point_coord(L.tx + 8 * j + 4, a.spacing_adiv));
    const float2 npyz = make_float2(-py, -pz);
    float2 tot[NJ];
#pragma unroll
    for (int j = 0; j < NJ; j++) tot[j] = make_float2(0.f, 0.f);

    // 32-bit shared address of the table, pre-biased so that the bit pattern of
    // (t + 2^23) rounded toward zero indexes it directly:
    // bits(t + 2^23) = 0x4B000000 + floor(t) for 0 <= t < 2^23.
    const uint32_t tab_base = (uint32_t)__cvta_generic_to_shared(s_tab4) - (MAGIC_BITS << 2);
    const float2 lom = make_float2(a.edge_lo, a.edge_lo), him = make_float2(a.edge_hi, a.edge_hi);
    uint32_t *bits = (MODE == FAR_TAB_TABLE && a.edge_bits) ? a.edge_bits + far_bits_base(a, f, chunk) + tid : nullptr;

    const int a_begin = chunk * a.chunk_atoms;
    const int a_end = min(a.n_atoms, a_begin + a.chunk_atoms);
    for (int a0 = a_begin; a0 < a_end; a0 += TILE) {
        const int na = min(TILE, a_end - a0);
        __syncthreads();
        for (int i = tid; i < TILE; i += EF_THREADS) {
            float4 v;
            if (i < na) {
                const int at = a0 + i;
                v.z = frame_atom_coord(__ldg(a.ax128 + at), X0);
                v.x = frame_atom_coord(__ldg(a.ay128 + at), Y0);
                v.y = frame_atom_coord(__ldg(a.az128 + at), Z0);
                v.w = __ldg(a.qw + at);
            } else {
                v = make_float4(0.f, 0.f, 0.f, 0.f);  // never read: the pair loops stop at na
            }
            s_atom[i] = v;
        }
        __syncthreads();
        if (!L.warp_in) continue;
        float2 acc[NJ];
#pragma unroll
        for (int j = 0; j < NJ; j++) acc[j] = make_float2(0.f, 0.f);
        if (MODE == FAR_TAB_CONST) {
            const float2 fT0 = make_float2(FAR_T0, FAR_T0);
#pragma unroll 2
            for (int i = 0; i < na; i++) {
                const float4 A = s_atom[i];
                const float2 dyz = __fadd2_rn(make_float2(A.x, A.y), npyz);
                const float s = __fmaf_rn(dyz.x, dyz.x, __fmaf_rn(dyz.y, dyz.y, TINY_T2));
                const float2 s2 = make_float2(s, s);
                const float2 ax2 = make_float2(A.z, A.z);
                const float2 q2 = make_float2(A.w, A.w);
#pragma unroll
                for (int j = 0; j < NJ; j++) {
                    const float2 dx = __fadd2_rn(ax2, npx[j]);
                    const float2 t2 = __ffma2_rn(dx, dx, s2);
                    const float2 rs = make_float2(rsqrt_approx(t2.x), rsqrt_approx(t2.y));
                    const float2 t = __fmul2_rn(t2, rs);
                    const float T0 = t.x < fT0.x ? 0.f : a.tab_const;
                    const float T1 = t.y < fT0.y ? 0.f : a.tab_const;
                    const float2 wv = __fmul2_rn(q2, rs);
                    acc[j] = __ffma2_rn(wv, make_float2(T0, T1), acc[j]);
                }
            }
        } else {
            const float2 tmax = make_float2(FAR_CLAMP_T, FAR_CLAMP_T);
            for (int ib = 0; ib < na; ib += 32) {
                const int nb = min(32, na - ib);
                uint32_t hist = 0;
#pragma unroll 2
                for (int ii = 0; ii < nb; ii++) {
                    const float4 A = s_atom[ib + ii];
                    const float2 dyz = __fadd2_rn(make_float2(A.x, A.y), npyz);
                    const float s = __fmaf_rn(dyz.x, dyz.x, __fmaf_rn(dyz.y, dyz.y, TINY_T2));
                    const float2 s2 = make_float2(s, s);
                    const float2 ax2 = make_float2(A.z, A.z);
                    const float2 q2 = make_float2(A.w, A.w);
                    uint32_t edge = 0;
#pragma unroll
                    for (int j = 0; j < NJ; j++) {
                        const float2 dx = __fadd2_rn(ax2, npx[j]);
                        const float2 t2 = __ffma2_rn(dx, dx, s2);
                        const float2 rs = make_float2(rsqrt_approx(t2.x), rsqrt_approx(t2.y));
                        float2 t = __fmul2_rn(t2, rs);
                        if (CLAMP) t = make_float2(fminf(t.x, tmax.x), fminf(t.y, tmax.y));
                        float2 lo, hi;
                        far_guard_bins(t, lom, him, lo, hi);
                        edge |= (__float_as_uint(lo.x) ^ __float_as_uint(hi.x)) |
                                (__float_as_uint(lo.y) ^ __float_as_uint(hi.y));
                        const float T0 = lds_f32(tab_base + (__float_as_uint(lo.x) << 2));
                        const float T1 = lds_f32(tab_base + (__float_as_uint(lo.y) << 2));
                        const float2 wv = __fmul2_rn(q2, rs);
                        acc[j] = __ffma2_rn(wv, make_float2(T0, T1), acc[j]);
                    }
                    hist = (hist << 1) | (edge ? 1u : 0u);
                }
                if (bits) bits[(size_t)((a0 - a_begin + ib) >> 5) * EF_THREADS] = hist << (32 - nb);  // atom k at bit 31-k
            }
        }
#pragma unroll
        for (int j = 0; j < NJ; j++) tot[j] = __fadd2_rn(tot[j], acc[j]);
    }

    const int iy = oy + L.ty, iz = oz + L.tz;
    if (iy < a.n1y && iz < a.n1z) {
        float *out = a.partial + (size_t)chunk * (size_t)a.P + ((size_t)iz * a.n1y + iy) * (size_t)a.n1x;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int ix0 = ox + L.tx + 8 * j, ix1 = ix0 + 4;
            if (ix0 < a.n1x) out[ix0] = tot[j].x;
            if (ix1 < a.n1x) out[ix1] = tot[j].y;
        }
    }
}

// The unit with as many x pairs as the frame has columns inside the box
// (CTA-uniform: only a box's last x frame can be partial), table mode and
// clamp of the instance (batch kernel).
template <int TILE, int MODE, bool CLAMP>
__device__ __forceinline__ void far_unit(const FarArgs &a, int f, int chunk, const float4 *s_tab4, float4 *s_atom)
{
    static_assert(EF_PAIRS == 4, "x-pair dispatch below");
    const int nj = (a.n1x - (f % a.nfx) * FRAME_X + 7) / 8;
    if (nj >= 4) far_unit_n<TILE, MODE, 4, CLAMP>(a, f, chunk, s_tab4, s_atom);
    else if (nj == 3) far_unit_n<TILE, MODE, 3, CLAMP>(a, f, chunk, s_tab4, s_atom);
    else if (nj == 2) far_unit_n<TILE, MODE, 2, CLAMP>(a, f, chunk, s_tab4, s_atom);
    else far_unit_n<TILE, MODE, 1, CLAMP>(a, f, chunk, s_tab4, s_atom);
}

template <int TILE>
__device__ __forceinline__ void far_dispatch(const FarArgs &a, int f, int chunk, const float4 *s_tab4, float4 *s_atom)
{
    if (a.tab_mode == FAR_TAB_CONST) far_unit<TILE, FAR_TAB_CONST, true>(a, f, chunk, s_tab4, s_atom);
    else if (a.clamp) far_unit<TILE, FAR_TAB_TABLE, true>(a, f, chunk, s_tab4, s_atom);
    else far_unit<TILE, FAR_TAB_TABLE, false>(a, f, chunk, s_tab4, s_atom);
}

// Single instance: one CTA per (frame, chunk) = (blockIdx.x, blockIdx.y).  The
// x-pair count of the box's last x frame (NJ_LAST) and the clamp are fixed per
// launch, so a grid whose last x frame is full compiles to the full-frame unit
// alone.
template <int TILE, int NJ_LAST, bool CLAMP>
__global__ void __launch_bounds__(EF_THREADS, 3) k_emap_far(FarArgs a)
{
    extern __shared__ float4 ef_smem[];
    float4 *s_tab4 = ef_smem;                     // a.tab_len floats
    float4 *s_atom = ef_smem + a.tab_len / 4;     // TILE entries
    if (a.tab_mode != FAR_TAB_CONST) load_far_table(s_tab4, a);
    __syncthreads();
    const int f = a.frame0 + blockIdx.x;
    const bool last = NJ_LAST < EF_PAIRS && f % a.nfx == a.nfx - 1;
    if (a.tab_mode == FAR_TAB_CONST) {
        if (last) far_unit_n<TILE, FAR_TAB_CONST, NJ_LAST, true>(a, f, blockIdx.y, s_tab4, s_atom);
        else far_unit_n<TILE, FAR_TAB_CONST, EF_PAIRS, true>(a, f, blockIdx.y, s_tab4, s_atom);
    } else {
        if (last) far_unit_n<TILE, FAR_TAB_TABLE, NJ_LAST, CLAMP>(a, f, blockIdx.y, s_tab4, s_atom);
        else far_unit_n<TILE, FAR_TAB_TABLE, EF_PAIRS, CLAMP>(a, f, blockIdx.y, s_tab4, s_atom);
    }
}

// ------------------------------------------------------------- fix-up ---
// The far pairs the guard flagged, resolved after the far-field kernel.  One
// CTA per far-field unit (frame, chunk), with the far kernel's lane layout.
// Each warp collects its threads' flagged (thread, atom) items from the edge
// bits into a shared list and processes them 32 at a time, one per lane:
// first the owner thread's pairs with that atom are re-evaluated by the far
// kernel's own FP32 operations (same inputs, same guard bins), giving the
// flagged pairs the owner keeps (t >= FAR_T0, point inside the box, bin below
// the last); then the lanes resolve those pairs one at a time together, each
// taking the exact bin from far_exact_bin and the correction
// w/r * (T_full[exact] - T_far[used]).  Corrections are summed per point in
// 64-bit fixed point (2^-40 kcal/mol units: integer addition, so the sum does
// not depend on which lane adds first) and added to the unit's partial sums.
// The e map therefore carries every far pair's reference bin, deterministically.
constexpr int FX_LIST = 64;                    // a warp's pending items: up to 32 appended to < 32 left
constexpr double FX_SCALE = 1099511627776.0;   // 2^40

struct FixSmem {
    float2 npx[EF_PAIRS][EF_THREADS];          // each thread's x pairs (negated frame coordinates)
    float2 npyz[EF_THREADS];
    unsigned long long corr[2 * EF_PAIRS][EF_THREADS];  // fixed-point corrections per point
    uint32_t items[EF_THREADS / 32][FX_LIST];  // (atom offset in the unit << 8) | owner thread
    // the frame's point coordinates in FP64 bins, (i - ne) * spacing * A_DIV:
    // x columns [0, FRAME_X), then y rows, then z planes
    double pc[FRAME_X + FRAME_Y + FRAME_Z];
    unsigned cnt[3];
};

// Exact bin of one flagged pair from FP64 coordinates already formed (the
// atom's x*A_DIV and the point's (i - ne) * spacing * A_DIV); see far_exact_bin.
__device__ __forceinline__ int far_exact_bin_d(double ax128, double ay128, double az128, double px, double py,
                                               double pz, int kb)
{
    const double dx = __dsub_rn(ax128, px);
    const double dy = __dsub_rn(ay128, py);
    const double dz = __dsub_rn(az128, pz);
    const double t2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    const double e = (double)(kb + 1), e2 = __dmul_rn(e, e);  // exact: kb < 2^23
    if (fabs(__dsub_rn(t2, e2)) > 1.0e-12 * e2) return t2 >= e2 ? kb + 1 : kb;
    const double inv = 1.0 / AG_A_DIV;  // exact
    const double r = hypot(__dmul_rn(dx, inv), hypot(__dmul_rn(dy, inv), __dmul_rn(dz, inv)));
    return (int)__dmul_rn(r, (double)AG_A_DIV) | FAR_TIE_FLAG;
}

// Per-lane tallies of the resolved pairs (summed once per unit).
struct FixCount {
    unsigned pairs, fp32_errors, ties;
};

// One (owner thread, atom) item: the owner's pairs with the atom re-evaluated
// by the far kernel's own FP32 operations (packed, as there), then each
// flagged pair the owner keeps (t >= FAR_T0, point inside the box, bin below
// the last) resolved in FP64 and its correction added.
template <int NJ, bool CLAMP>
__device__ __forceinline__ void far_fix_item(const FarArgs &a, FixSmem &S, uint32_t item, int a_begin, int ox, int oy,
                                             int oz, double X0, double Y0, double Z0, FixCount &n)
{
    const int owner = (int)(item & 255u), at = a_begin + (int)(item >> 8);
    const int lane = owner & 31, w = owner >> 5;
    const int tx = lane & 3, ty = ((lane >> 2) & 3) + 4 * (w & 1), tz = (lane >> 4) + 2 * (w >> 1);
    const double ax128 = __ldg(a.ax128 + at), ay128 = __ldg(a.ay128 + at), az128 = __ldg(a.az128 + at);
    const float ax = frame_atom_coord(ax128, X0), ay = frame_atom_coord(ay128, Y0), az = frame_atom_coord(az128, Z0);
    const float qa = __ldg(a.qw + at);
    const float2 dyz = __fadd2_rn(make_float2(ay, az), S.npyz[owner]);
    const float s = __fmaf_rn(dyz.x, dyz.x, __fmaf_rn(dyz.y, dyz.y, TINY_T2));
    const float2 s2 = make_float2(s, s), ax2 = make_float2(ax, ax);
    const float2 tmax = make_float2(FAR_CLAMP_T, FAR_CLAMP_T);
    const float2 lom = make_float2(a.edge_lo, a.edge_lo), him = make_float2(a.edge_hi, a.edge_hi);
    const float2 fT0 = make_float2(FAR_T0, FAR_T0);
    // the owner's flagged pairs with this atom (slot 2j + c: x = tx + 8j + 4c):
    // the guard bins alone; the rare flagged pairs the owner does not keep
    // are dropped below, one at a time
    uint32_t mask = 0;
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        const float2 dx = __fadd2_rn(ax2, S.npx[j][owner]);
        const float2 t2 = __ffma2_rn(dx, dx, s2);
        float2 t = __fmul2_rn(t2, make_float2(rsqrt_approx(t2.x), rsqrt_approx(t2.y)));
        if (CLAMP) t = make_float2(fminf(t.x, tmax.x), fminf(t.y, tmax.y));
        float2 lo, hi;
        far_guard_bins(t, lom, him, lo, hi);
        mask |= min(__float_as_uint(lo.x) ^ __float_as_uint(hi.x), 1u) << (2 * j);
        mask |= min(__float_as_uint(lo.y) ^ __float_as_uint(hi.y), 1u) << (2 * j + 1);
    }
    while (mask) {
        const int sl = __ffs(mask) - 1;
        mask &= mask - 1;
        // the pair again, scalar (the same operations component-wise)
        const float2 npx2 = S.npx[sl >> 1][owner];
        const float dx = __fadd_rn(ax, (sl & 1) ? npx2.y : npx2.x);
        const float t2 = __fmaf_rn(dx, dx, s);
        const float rs = rsqrt_approx(t2);
        float t = __fmul_rn(t2, rs);
        if (CLAMP) t = fminf(t, FAR_CLAMP_T);
        const uint32_t bl = __float_as_uint(__fmaf_rz(t, a.edge_lo, 8388608.f));
        const int kb = (int)(bl - MAGIC_BITS);
        const int ix = ox + tx + 8 * (sl >> 1) + 4 * (sl & 1);
        // the owner keeps pairs at t >= FAR_T0 (nearer ones are the near
        // kernel's), at points inside the box, below the last bin (there the
        // reference clamps too)
        if (!(t >= fT0.x) || ix >= a.n1x || kb >= AG_NDIEL - 1) continue;
        const int kr = far_exact_bin_d(ax128, ay128, az128, S.pc[ix - ox], S.pc[FRAME_X + ty], S.pc[FRAME_X + FRAME_Y + tz],
                                       kb);
        const int kx = kr & ~FAR_TIE_FLAG;
        const int kf = (int)(__float_as_uint(__fadd_rz(t, 8388608.f)) - MAGIC_BITS);  // plain FP32 floor(t)
        n.pairs++;
        n.fp32_errors += min(kf, AG_NDIEL - 1) != kx ? 1u : 0u;
        n.ties += (kr & FAR_TIE_FLAG) ? 1u : 0u;
        // the far kernel added T_far[kb]; T_far is zero below FAR_BIN0, so an
        // owned pair whose exact bin is 1023 needs T[1023] even when kx == kb
        const float used = __ldg(a.far_tab + kb);
        const float dT = __fsub_rn(__ldg(a.tab_full + min(kx, AG_NDIEL - 1)), used);
        if (dT != 0.f) {
            // scaling by 2^40 is exact in FP32 as in FP64 (no overflow or
            // underflow at these magnitudes), so the float product is rounded once
            const float v = __fmul_rn(__fmul_rn(__fmul_rn(qa, rs), dT), (float)FX_SCALE);
            atomicAdd(&S.corr[sl][owner], (unsigned long long)__float2ll_rn(v));
        }
    }
}

template <int NJ, bool CLAMP>
__device__ __forceinline__ void far_fix_unit(const FarArgs &a, int f, int chunk, FixSmem &S)
{
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int fx = f % a.nfx, fy = (f / a.nfx) % a.nfy, fz = f / (a.nfx * a.nfy);
    const int ox = fx * FRAME_X, oy = fy * FRAME_Y, oz = fz * FRAME_Z;
    const double X0 = frame_origin_bins(ox, a.nex, a.spacing_adiv);
    const double Y0 = frame_origin_bins(oy, a.ney, a.spacing_adiv);
    const double Z0 = frame_origin_bins(oz, a.nez, a.spacing_adiv);
    const FarLane L = far_lane(a, tid, oy, oz);
    const bool point_in = oy + L.ty < a.n1y && oz + L.tz < a.n1z;
    __syncthreads();  // the previous unit (batch kernel) is done with S
#pragma unroll
    for (int j = 0; j < EF_PAIRS; j++) {
        S.npx[j][tid] = make_float2(-frame_point_coord(L.tx + 8 * j, a.spacing_adiv),
                                    -frame_point_coord(L.tx + 8 * j + 4, a.spacing_adiv));
        S.corr[2 * j][tid] = 0ull;
        S.corr[2 * j + 1][tid] = 0ull;
    }
    S.npyz[tid] = make_float2(-frame_point_coord(L.ty, a.spacing_adiv), -frame_point_coord(L.tz, a.spacing_adiv));
    if (tid < FRAME_X + FRAME_Y + FRAME_Z) {
        const int i = tid < FRAME_X ? ox + tid - a.nex
                    : tid < FRAME_X + FRAME_Y ? oy + (tid - FRAME_X) - a.ney : oz + (tid - FRAME_X - FRAME_Y) - a.nez;
        S.pc[tid] = __dmul_rn((double)i, a.spacing_adiv);
    }
    if (tid < 3) S.cnt[tid] = 0u;
    __syncthreads();
    const int a_begin = chunk * a.chunk_atoms;
    const int a_end = min(a.n_atoms, a_begin + a.chunk_atoms);
    const int nwords = (a_end - a_begin + 31) >> 5;
    const uint32_t *bits = a.edge_bits + far_bits_base(a, f, chunk) + tid;
    uint32_t *list = S.items[w];
    FixCount cnt = {0u, 0u, 0u};
    if (L.warp_in) {  // the far kernel wrote no words for the other warps
        int nlist = 0;  // warp-uniform: pending items in list[0, nlist)
        const unsigned below = (1u << lane) - 1u;
        for (int k = 0; k < nwords; k++) {
            // points past the box are neither written nor fixed
            uint32_t h = point_in ? __ldg(bits + (size_t)k * EF_THREADS) : 0u;
            // append the word's items, at most one per lane per step, and run
            // a round of 32 whenever 32 are pending
            for (;;) {
                const unsigned have = __ballot_sync(0xffffffffu, h != 0u);
                if (!have) break;
                if (h) {
                    const int b = __clz(h);
                    h &= ~(0x80000000u >> b);
                    list[nlist + __popc(have & below)] = ((uint32_t)(32 * k + b) << 8) | (uint32_t)tid;
                }
                nlist += __popc(have);
                if (nlist >= 32) {  // warp-uniform; the appends become visible here
                    __syncwarp();
                    far_fix_item<NJ, CLAMP>(a, S, list[lane], a_begin, ox, oy, oz, X0, Y0, Z0, cnt);
                    nlist -= 32;
                    const uint32_t rest = lane < nlist ? list[32 + lane] : 0u;
                    __syncwarp();
                    if (lane < nlist) list[lane] = rest;
                    __syncwarp();
                }
            }
        }
        __syncwarp();
        if (lane < nlist) far_fix_item<NJ, CLAMP>(a, S, list[lane], a_begin, ox, oy, oz, X0, Y0, Z0, cnt);
    }
    __syncwarp();
    // each thread adds its own points' corrections to the unit's partial sums
    const int iy = oy + L.ty, iz = oz + L.tz;
    if (L.warp_in && point_in) {
        float *out = a.partial + (size_t)chunk * (size_t)a.P + ((size_t)iz * a.n1y + iy) * (size_t)a.n1x;
#pragma unroll
        for (int j = 0; j < NJ; j++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const long long v = (long long)S.corr[2 * j + c][tid];
                const int ix = ox + L.tx + 8 * j + 4 * c;
                if (v != 0 && ix < a.n1x) out[ix] = __fadd_rn(out[ix], (float)((double)v / FX_SCALE));
            }
    }
    const unsigned c0 = __reduce_add_sync(0xffffffffu, cnt.pairs);
    const unsigned c1 = __reduce_add_sync(0xffffffffu, cnt.fp32_errors);
    const unsigned c2 = __reduce_add_sync(0xffffffffu, cnt.ties);
    if (lane == 0 && (c0 | c1 | c2)) {
        atomicAdd(&S.cnt[0], c0);
        atomicAdd(&S.cnt[1], c1);
        atomicAdd(&S.cnt[2], c2);
    }
    __syncthreads();
    if (tid < 3 && a.edge_counters && S.cnt[tid]) atomicAdd(a.edge_counters + tid, (unsigned long long)S.cnt[tid]);
}

template <bool CLAMP>
__device__ __forceinline__ void far_fix_nj(const FarArgs &a, int f, int chunk, FixSmem &S)
{
    const int nj = (a.n1x - (f % a.nfx) * FRAME_X + 7) / 8;
    if (nj >= 4) far_fix_unit<4, CLAMP>(a, f, chunk, S);
    else if (nj == 3) far_fix_unit<3, CLAMP>(a, f, chunk, S);
    else if (nj == 2) far_fix_unit<2, CLAMP>(a, f, chunk, S);
    else far_fix_unit<1, CLAMP>(a, f, chunk, S);
}

__device__ __forceinline__ void far_fix_dispatch(const FarArgs &a, int f, int chunk, FixSmem &S)
{
    if (a.clamp) far_fix_nj<true>(a, f, chunk, S);
    else far_fix_nj<false>(a, f, chunk, S);
}

// Single instance: one CTA per (frame, chunk), frames from a.frame0.
__global__ void __launch_bounds__(EF_THREADS) k_far_fixup(FarArgs a)
{
    extern __shared__ float4 fx_smem[];
    FixSmem &S = *(FixSmem *)fx_smem;
    // read through a shared copy: a reference to the parameter would be
    // copied to local memory by every thread
    __shared__ FarArgs s_a;
    if (threadIdx.x == 0) s_a = a;
    __syncthreads();
    far_fix_dispatch(s_a, s_a.frame0 + blockIdx.x, blockIdx.y, S);
}

// Many instances: one CTA per unit of any instance (unit_begin as the batch
// far kernel numbers them); instances without a far-field table get none.
__global__ void __launch_bounds__(EF_THREADS) k_far_fixup_batch(const FarArgs *__restrict__ insts,
                                                                const long long *__restrict__ unit_begin, int n_inst)
{
    extern __shared__ float4 fx_smem[];
    FixSmem &S = *(FixSmem *)fx_smem;
    __shared__ FarArgs s_a;
    const long long u = (long long)blockIdx.x + ((long long)blockIdx.y << 31);
    if (u >= unit_begin[n_inst]) return;
    int lo = 0, hi = n_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (unit_begin[mid] <= u) lo = mid; else hi = mid - 1;
    }
    if (threadIdx.x == 0) s_a = insts[lo];
    __syncthreads();
    if (s_a.tab_mode == FAR_TAB_CONST || !s_a.edge_bits) return;
    const long long lu = u - unit_begin[lo];
    const int frames = s_a.nfx * s_a.nfy * s_a.nfz;
    far_fix_dispatch(s_a, (int)(lu % frames), (int)(lu / frames), S);
}

// Many instances, persistent: each CTA takes (instance, frame, chunk) units
// from an atomic counter until none is left; units are numbered instance by
// instance (instances ordered by decreasing work) and never wait on each other.
// The dynamic shared memory holds the longest table of the batch and a tile.
template <int TILE>
__global__ void __launch_bounds__(EF_THREADS, 3)
k_emap_far_batch(const FarArgs *__restrict__ insts, const long long *__restrict__ unit_begin, int n_inst,
                 unsigned long long *__restrict__ counter, int max_tab_len)
{
    extern __shared__ float4 ef_smem[];
    float4 *s_tab4 = ef_smem;
    float4 *s_atom = ef_smem + max_tab_len / 4;
    __shared__ long long s_unit;
    __shared__ FarArgs s_a;
    int cur = -1;
    const long long total = unit_begin[n_inst];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_unit = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long u = s_unit;
        if (u >= total) break;
        int lo = 0, hi = n_inst - 1;  // instance holding unit u
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (unit_begin[mid] <= u) lo = mid; else hi = mid - 1;
        }
        if (lo != cur) {
            __syncthreads();
            if (threadIdx.x == 0) s_a = insts[lo];
            __syncthreads();
            if (s_a.tab_mode != FAR_TAB_CONST) load_far_table(s_tab4, s_a);
            cur = lo;
        }
        const long long lu = u - unit_begin[lo];
        const int frames = s_a.nfx * s_a.nfy * s_a.nfz;
        const int fr = (int)(lu % frames), ch = (int)(lu / frames);
        far_dispatch<TILE>(s_a, fr, ch, s_tab4, s_atom);
    }
}

// Bins of the far field for every (listed point, atom) pair, with the far
// kernel's own arithmetic (frame-relative FP32 coordinates of the point's
// frame, guard bins, far_exact_bin): used[k] = the bin the far kernel's
// result carries for the pair (-1 for a near-field pair, t < FAR_T0),
// fp32[k] = floor(t) of the FP32 distance, flags[k] = 1 when the guard bins
// differ (resolved in FP64), | 2 when that resolution was a tie.  k = point
// slot * n_atoms + atom.  A diagnostic for tests on small problems.
__global__ void __launch_bounds__(256) k_far_bins_debug(FarArgs a, const long long *__restrict__ pts, int n_pts,
                                                        int *__restrict__ used, int *__restrict__ fp32,
                                                        int *__restrict__ flags)
{
    const long long k = (long long)blockIdx.x * 256 + threadIdx.x;
    if (k >= (long long)n_pts * a.n_atoms) return;
    const int at = (int)(k % a.n_atoms);
    const long long lin = pts[k / a.n_atoms];
    const int ix = (int)(lin % a.n1x), iy = (int)((lin / a.n1x) % a.n1y), iz = (int)(lin / ((long long)a.n1x * a.n1y));
    const int ox = ix / FRAME_X * FRAME_X, oy = iy / FRAME_Y * FRAME_Y, oz = iz / FRAME_Z * FRAME_Z;
    const float ax = frame_atom_coord(a.ax128[at], frame_origin_bins(ox, a.nex, a.spacing_adiv));
    const float ay = frame_atom_coord(a.ay128[at], frame_origin_bins(oy, a.ney, a.spacing_adiv));
    const float az = frame_atom_coord(a.az128[at], frame_origin_bins(oz, a.nez, a.spacing_adiv));
    const float s = far_pair_s(ay, az, frame_point_coord(iy - oy, a.spacing_adiv),
                               frame_point_coord(iz - oz, a.spacing_adiv));
    const float t = fminf(far_pair_t(ax, frame_point_coord(ix - ox, a.spacing_adiv), s), FAR_CLAMP_T);
    const int kl = (int)(__float_as_uint(__fmaf_rz(t, a.edge_lo, 8388608.f)) - MAGIC_BITS);
    const int kh = (int)(__float_as_uint(__fmaf_rz(t, a.edge_hi, 8388608.f)) - MAGIC_BITS);
    fp32[k] = (int)(__float_as_uint(__fadd_rz(t, 8388608.f)) - MAGIC_BITS);
    int u = kl, fl = 0;
    if (kl != kh) {
        fl = 1;
        if (t >= FAR_T0) {
            const int kr = far_exact_bin(a.ax128, a.ay128, a.az128, at, a.spacing_adiv, ix - a.nex, iy - a.ney,
                                         iz - a.nez, kl);
            u = kr & ~FAR_TIE_FLAG;
            if (kr & FAR_TIE_FLAG) fl |= 2;
        }
    }
    used[k] = t >= FAR_T0 ? min(u, AG_NDIEL - 1) : -1;
    flags[k] = fl;
}

cudaError_t launch_far_bins_debug(const FarArgs &a, const long long *pts, int n_pts, int *used, int *fp32, int *flags,
                                  cudaStream_t s)
{
    const long long n = (long long)n_pts * a.n_atoms;
    if (n <= 0) return cudaSuccess;
    k_far_bins_debug<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, pts, n_pts, used, fp32, flags);
    return cudaGetLastError();
}

// FP64 twin of LOOP 1: one thread per point, all atoms in file order.
constexpr int EX_THREADS = 128;
constexpr int EX_TILE = 256;

__global__ void __launch_bounds__(EX_THREADS)
k_emap_exact(DevProblem p, double *__restrict__ emap)
{
    __shared__ double s_x[EX_TILE], s_y[EX_TILE], s_z[EX_TILE], s_q[EX_TILE];
    const long long lin = (long long)blockIdx.x * EX_THREADS + threadIdx.x;
    const bool valid = lin < p.P;
    const int ix = (int)(lin % p.n1x), iy = (int)((lin / p.n1x) % p.n1y), iz = (int)(lin / ((long long)p.n1x * p.n1y));
    const double cx = (double)(ix - p.nex) * p.spacing;
    const double cy = (double)(iy - p.ney) * p.spacing;
    const double cz = (double)(iz - p.nez) * p.spacing;
    double e = 0.0;
    for (int a0 = 0; a0 < p.n_atoms; a0 += EX_TILE) {
        const int na = min(EX_TILE, p.n_atoms - a0);
        __syncthreads();
        for (int i = threadIdx.x; i < na; i += EX_THREADS) {
            s_x[i] = p.x[a0 + i]; s_y[i] = p.y[a0 + i]; s_z[i] = p.z[a0 + i]; s_q[i] = p.q[a0 + i];
        }
        __syncthreads();
        for (int i = 0; i < na; i++) {
            double r = hypot(__dsub_rn(s_x[i], cx), hypot(__dsub_rn(s_y[i], cy), __dsub_rn(s_z[i], cz)));
            if (r < 1.0e-6) r = 1.0e-6;
            const double inv_rmax = __ddiv_rn(1.0, r > 0.5 ? r : 0.5);
            int k = (int)__dmul_rn(r, (double)AG_A_DIV);
            if (k > AG_NDIEL - 1) k = AG_NDIEL - 1;
            const double f = p.dddiel ? p.reps[k] : p.invdielcal;
            e = __dadd_rn(e, __dmul_rn(__dmul_rn(__dmul_rn(s_q[i], inv_rmax), f), p.coeff_estat));
        }
    }
    if (valid) emap[lin] = e;
}

}  // namespace agb

namespace agb {

int frames_x(int n1x) { return (n1x + FRAME_X - 1) / FRAME_X; }
int frames_y(int n1y) { return (n1y + FRAME_Y - 1) / FRAME_Y; }
int frames_z(int n1z) { return (n1z + FRAME_Z - 1) / FRAME_Z; }

size_t far_smem_bytes(int tile, int tab_len) { return (size_t)tab_len * sizeof(float) + (size_t)tile * sizeof(float4); }

int far_edge_words(int chunk_atoms) { return (std::max(chunk_atoms, 1) + 31) / 32; }

size_t far_edge_bits_bytes(int n_chunks, int chunk_atoms, int nframes)
{
    return (size_t)std::max(n_chunks, 0) * (size_t)std::max(nframes, 0) * (size_t)far_edge_words(chunk_atoms) *
           EF_THREADS * sizeof(uint32_t);
}

cudaError_t launch_far_fixup(const FarArgs &args, int n_chunks, cudaStream_t s, int fz0, int fz1)
{
    if (args.tab_mode == FAR_TAB_CONST || !args.edge_bits || n_chunks <= 0) return cudaSuccess;
    FarArgs a = args;
    if (fz1 < 0 || fz1 > a.nfz) fz1 = a.nfz;
    if (fz0 >= fz1) return cudaSuccess;
    a.frame0 = fz0 * a.nfx * a.nfy;
    dim3 grid((unsigned)(a.nfx * a.nfy * (fz1 - fz0)), (unsigned)n_chunks);
    k_far_fixup<<<grid, EF_THREADS, sizeof(FixSmem), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_far_fixup_batch(const FarArgs *insts, const long long *unit_begin, int n_inst, long long n_units,
                                   cudaStream_t s)
{
    if (n_inst <= 0 || n_units <= 0) return cudaSuccess;
    const long long gx = std::min<long long>(n_units, (1LL << 31) - 1);
    const long long gy = (n_units + (1LL << 31) - 1) >> 31;
    k_far_fixup_batch<<<dim3((unsigned)gx, (unsigned)gy), EF_THREADS, sizeof(FixSmem), s>>>(insts, unit_begin, n_inst);
    return cudaGetLastError();
}

// Frame z-rows [fz0, fz1) of one instance (fz1 < 0: through the last).
template <bool CLAMP>
static void far_launch_nj(const FarArgs &a, dim3 grid, size_t smem, cudaStream_t s)
{
    const int nj_last = (a.n1x - (a.nfx - 1) * FRAME_X + 7) / 8;  // x pairs of the last frame inside the box
    if (nj_last >= 4) k_emap_far<512, 4, CLAMP><<<grid, EF_THREADS, smem, s>>>(a);
    else if (nj_last == 3) k_emap_far<512, 3, CLAMP><<<grid, EF_THREADS, smem, s>>>(a);
    else if (nj_last == 2) k_emap_far<512, 2, CLAMP><<<grid, EF_THREADS, smem, s>>>(a);
    else k_emap_far<512, 1, CLAMP><<<grid, EF_THREADS, smem, s>>>(a);
}

cudaError_t launch_emap_far(const FarArgs &args, int n_chunks, int tile, cudaStream_t s, int fz0, int fz1)
{
    if (tile != 512) return cudaErrorInvalidValue;  // the single-instance kernel stages 512-atom tiles
    if (args.tab_len < 0 || args.tab_len > FAR_TAB_MAX || args.tab_len % 4) return cudaErrorInvalidValue;
    FarArgs a = args;
    if (fz1 < 0 || fz1 > a.nfz) fz1 = a.nfz;
    if (fz0 >= fz1) return cudaSuccess;
    a.frame0 = fz0 * a.nfx * a.nfy;
    dim3 grid((unsigned)(a.nfx * a.nfy * (fz1 - fz0)), (unsigned)n_chunks);
    const size_t smem = far_smem_bytes(512, a.tab_len);
    if (a.clamp || a.tab_mode == FAR_TAB_CONST) far_launch_nj<true>(a, grid, smem, s);
    else far_launch_nj<false>(a, grid, smem, s);
    return cudaGetLastError();
}

int current_device_sms()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0)
        return 148;
    return sms;
}

cudaError_t prepare_far_kernels()
{
    const int s512 = (int)far_smem_bytes(512, FAR_TAB_MAX);
    const void *single[] = {(const void *)k_emap_far<512, 1, true>, (const void *)k_emap_far<512, 2, true>,
                            (const void *)k_emap_far<512, 3, true>, (const void *)k_emap_far<512, 4, true>,
                            (const void *)k_emap_far<512, 1, false>, (const void *)k_emap_far<512, 2, false>,
                            (const void *)k_emap_far<512, 3, false>, (const void *)k_emap_far<512, 4, false>};
    for (const void *fn : single) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, s512);
        if (e != cudaSuccess) return e;
    }
    for (const void *fn : {(const void *)k_far_fixup, (const void *)k_far_fixup_batch}) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FixSmem));
        if (e != cudaSuccess) return e;
    }
    const void *batch[] = {(const void *)k_emap_far_batch<256>, (const void *)k_emap_far_batch<512>,
                           (const void *)k_emap_far_batch<1024>};
    const int tiles[] = {256, 512, 1024};
    for (int k = 0; k < 3; k++) {
        cudaError_t e = cudaFuncSetAttribute(batch[k], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)far_smem_bytes(tiles[k], FAR_TAB_MAX));
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The persistent batch kernel: as many CTAs as fit (at most ctas_per_sm) on
// every SM.  Its shared-memory limit is set by prepare_far_kernels().
template <int TILE>
static cudaError_t far_batch_t(const FarArgs *insts, const long long *unit_begin, int n_inst,
                               unsigned long long *counter, int ctas_per_sm, int max_tab_len, cudaStream_t s)
{
    const size_t smem = far_smem_bytes(TILE, max_tab_len);
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_emap_far_batch<TILE>, EF_THREADS, smem);
    if (e != cudaSuccess) return e;
    const int per_sm = std::max(1, std::min(ctas_per_sm, occ));
    k_emap_far_batch<TILE><<<current_device_sms() * per_sm, EF_THREADS, smem, s>>>(insts, unit_begin, n_inst, counter,
                                                                                   max_tab_len);
    return cudaGetLastError();
}

cudaError_t launch_emap_far_batch(const FarArgs *insts, const long long *unit_begin, int n_inst,
                                  unsigned long long *counter, int tile, int ctas_per_sm, int max_tab_len,
                                  cudaStream_t s)
{
    if (max_tab_len < 0 || max_tab_len > FAR_TAB_MAX || max_tab_len % 4) return cudaErrorInvalidValue;
    if (tile == 256) return far_batch_t<256>(insts, unit_begin, n_inst, counter, ctas_per_sm, max_tab_len, s);
    if (tile == 1024) return far_batch_t<1024>(insts, unit_begin, n_inst, counter, ctas_per_sm, max_tab_len, s);
    return far_batch_t<512>(insts, unit_begin, n_inst, counter, ctas_per_sm, max_tab_len, s);
}

// One thread per point of every instance: instance i owns points
// [begin[i], begin[i+1]) of the flattened range.
__global__ void __launch_bounds__(256) k_emap_reduce(const ReduceInst *__restrict__ insts,
                                                     const long long *__restrict__ begin, int n)
{
    const long long total = begin[n];
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < total;
         u += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (begin[mid] <= u) lo = mid;
            else hi = mid - 1;
        }
        const ReduceInst r = insts[lo];
        const long long lin = u - begin[lo];
        float e = 0.f;
        for (int c = 0; c < r.n_chunks; c++) e += r.partial[(size_t)c * (size_t)r.P + (size_t)lin];
        r.out[lin] = e + r.out[lin];
    }
}

// Points [lin0, lin1) of one instance.
__global__ void __launch_bounds__(256) k_emap_reduce_range(ReduceInst r, long long lin0, long long lin1)
{
    for (long long lin = lin0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; lin < lin1;
         lin += (long long)gridDim.x * blockDim.x) {
        float e = 0.f;
        for (int c = 0; c < r.n_chunks; c++) e += r.partial[(size_t)c * (size_t)r.P + (size_t)lin];
        r.out[lin] = e + r.out[lin];
    }
}

cudaError_t launch_emap_reduce_range(const ReduceInst &r, long long lin0, long long lin1, cudaStream_t s)
{
    if (lin1 <= lin0) return cudaSuccess;
    const unsigned nb = (unsigned)std::min<long long>((lin1 - lin0 + 255) / 256, 16LL * current_device_sms());
    k_emap_reduce_range<<<nb, 256, 0, s>>>(r, lin0, lin1);
    return cudaGetLastError();
}

cudaError_t launch_emap_reduce(const ReduceInst *insts, const long long *begin, int n, long long total,
                               cudaStream_t s)
{
    if (n <= 0 || total <= 0) return cudaSuccess;
    const long long want = (total + 255) / 256;
    const unsigned nb = (unsigned)std::min<long long>(want, 16LL * current_device_sms());
    k_emap_reduce<<<nb, 256, 0, s>>>(insts, begin, n);
    return cudaGetLastError();
}

cudaError_t launch_emap_exact(const DevProblem &p, double *emap, cudaStream_t s)
{
    const unsigned nb = (unsigned)((p.P + EX_THREADS - 1) / EX_THREADS);
    k_emap_exact<<<nb, EX_THREADS, 0, s>>>(p, emap);
    return cudaGetLastError();
}

}  // namespace agb
