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

__device__ __forceinline__ void load_far_table(float4 *s_tab4, const float *far_tab)
{
    for (int i = threadIdx.x; i < AG_NDIEL / 4; i += EF_THREADS) s_tab4[i] = __ldg(((const float4 *)far_tab) + i);
}

// Exact LOOP 1 bin of a far pair whose guard bins differ (kb and kb + 1):
// the reference's bin (int)(r*A_DIV) with r = hypot(dx, hypot(dy, dz))
// (main.cpp:97, :2951-2956).  The FP64 differences are the reference's
// coordinate differences scaled by A_DIV = 2^7 (exact: x*A_DIV, and the grid
// coordinate ((i - ne)*spacing)*A_DIV = (i - ne)*(spacing*A_DIV); ix, iy, iz
// are i - ne); the squared distance decides against the edge (kb + 1)^2
// unless it lies within 1e-12 of it, where the reference's own expression
// decides and the result carries FAR_TIE_FLAG.  Scalars only: a struct
// argument of a non-inlined function would be copied to local memory.
__device__ __noinline__ int far_exact_bin(const double *ax128, const double *ay128, const double *az128, int at,
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

// One work unit: frame `f` of one instance against atom chunk `chunk`.
// The caller has loaded the instance's table into s_tab4 and synchronised.
// Atom tile entries: frame-relative X, Y, Z in bins and w = q*coeff_estat*A_DIV.
// The first NJ pairs of each thread hold the frame's x columns inside the box
// (the rest is padding and is skipped), and a warp whose 4 rows or 2 planes
// all lie past the box skips the pairs.
//
// Table bins (FAR_TAB_TABLE).  Each pair's table value is T[floor(t*edge_lo)];
// a pair whose second guard bin floor(t*edge_hi) differs lies within the FP32
// error bound of a bin edge.  Each thread records, per block of 32 atoms, a
// bit per atom with such a pair among its own (s_hist); after the tile it
// re-evaluates the pairs of those atoms with the same FP32 operations, takes
// the exact bin of each flagged pair it owns (t >= FAR_T0) from far_exact_bin
// and adds w/r * (T[exact] - T[used]) to its own point.  The bins of every far
// pair are therefore the reference's, and the result stays deterministic.
template <int MODE, int NJ>
__device__ __forceinline__ void far_fix_atom(const FarArgs &a, const float4 A, int at, const float2 *npx, float2 npyz,
                                             float2 lom, float2 him, uint32_t tab_base, int ox, int iy, int iz, int tx,
                                             float2 *tot, unsigned *s_cnt)
{
    const float2 dyz = __fadd2_rn(make_float2(A.y, A.z), npyz);
    const float s = __fmaf_rn(dyz.x, dyz.x, __fmaf_rn(dyz.y, dyz.y, TINY_T2));
    const float2 s2 = make_float2(s, s);
    const float2 ax2 = make_float2(A.x, A.x);
    const float2 q2 = make_float2(A.w, A.w);
    const float2 tmax = make_float2(FAR_CLAMP_T, FAR_CLAMP_T);
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        const float2 dx = __fadd2_rn(ax2, npx[j]);
        const float2 t2 = __ffma2_rn(dx, dx, s2);
        const float2 rs = make_float2(rsqrt_approx(t2.x), rsqrt_approx(t2.y));
        float2 t = __fmul2_rn(t2, rs);
        t = make_float2(fminf(t.x, tmax.x), fminf(t.y, tmax.y));
        float2 lo, hi;
        far_guard_bins(t, lom, him, lo, hi);
        const float2 wv = __fmul2_rn(q2, rs);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const float tc = c ? t.y : t.x;
            const uint32_t bl = __float_as_uint(c ? lo.y : lo.x), bh = __float_as_uint(c ? hi.y : hi.x);
            const int ix = ox + tx + 8 * j + 4 * c;
            if (bl == bh || !(tc >= FAR_T0) || ix >= a.n1x) continue;  // unflagged, near-field, or past the box
            const int kb = (int)(bl - MAGIC_BITS);
            const int kr = far_exact_bin(a.ax128, a.ay128, a.az128, at, a.spacing_adiv, ix - a.nex, iy - a.ney,
                                         iz - a.nez, kb);
            const int kx = kr & ~FAR_TIE_FLAG;
            const int kf = (int)(__float_as_uint(__fadd_rz(tc, 8388608.f)) - MAGIC_BITS);  // plain FP32 floor(t)
            atomicAdd(s_cnt, 1u);
            if (kf != kx) atomicAdd(s_cnt + 1, 1u);
            if (kr & FAR_TIE_FLAG) atomicAdd(s_cnt + 2, 1u);
            if (kx != kb) {
                const float used = lds_f32(tab_base + (bl << 2));
                const float dT = __fsub_rn(__ldg(a.tab_full + min(kx, AG_NDIEL - 1)), used);
                if (c) tot[j].y = __fmaf_rn(wv.y, dT, tot[j].y);
                else tot[j].x = __fmaf_rn(wv.x, dT, tot[j].x);
            }
        }
    }
}

// s_cnt: three shared counters of the CTA (far_fix_atom), zero on entry;
// the unit adds them to a.edge_counters and leaves them zero.
template <int TILE, int MODE, int NJ>
__device__ __forceinline__ void far_unit_n(const FarArgs &a, int f, int chunk, const float4 *s_tab4, float4 *s_atom,
                                           uint32_t *s_hist, unsigned *s_cnt)
{
    const int tid = threadIdx.x;
    const int fx = f % a.nfx, fy = (f / a.nfx) % a.nfy, fz = f / (a.nfx * a.nfy);
    const int ox = fx * FRAME_X, oy = fy * FRAME_Y, oz = fz * FRAME_Z;
    // frame origin in bins, exactly (ox-nex)*spacing*A_DIV as the reference forms c (main.cpp:2859)
    const double X0 = frame_origin_bins(ox, a.nex, a.spacing_adiv);
    const double Y0 = frame_origin_bins(oy, a.ney, a.spacing_adiv);
    const double Z0 = frame_origin_bins(oz, a.nez, a.spacing_adiv);

    // compact 4x4x2 lane footprint per warp (fewest table bank conflicts)
    const int lane = tid & 31, w = tid >> 5;
    const int tx = lane & 3;
    const int ty = ((lane >> 2) & 3) + 4 * (w & 1);
    const int tz = (lane >> 4) + 2 * (w >> 1);
    const bool warp_in = oy + 4 * (w & 1) < a.n1y && oz + 2 * (w >> 1) < a.n1z;
    const float py = frame_point_coord(ty, a.spacing_adiv);
    const float pz = frame_point_coord(tz, a.spacing_adiv);
    float2 npx[NJ];
#pragma unroll
    for (int j = 0; j < NJ; j++)
        npx[j] = make_float2(-frame_point_coord(tx + 8 * j, a.spacing_adiv),
                             -frame_point_coord(tx + 8 * j + 4, a.spacing_adiv));
    const float2 npyz = make_float2(-py, -pz);
    float2 tot[NJ];
#pragma unroll
    for (int j = 0; j < NJ; j++) tot[j] = make_float2(0.f, 0.f);

    // 32-bit shared address of the table, pre-biased so that the bit pattern of
    // (t + 2^23) rounded toward zero indexes it directly:
    // bits(t + 2^23) = 0x4B000000 + floor(t) for 0 <= t < 2^23.
    const uint32_t tab_base = (uint32_t)__cvta_generic_to_shared(s_tab4) - (MAGIC_BITS << 2);
    const float2 lom = make_float2(a.edge_lo, a.edge_lo), him = make_float2(a.edge_hi, a.edge_hi);

    const int a_begin = chunk * a.chunk_atoms;
    const int a_end = min(a.n_atoms, a_begin + a.chunk_atoms);
    for (int a0 = a_begin; a0 < a_end; a0 += TILE) {
        const int na = min(TILE, a_end - a0);
        __syncthreads();
        for (int i = tid; i < TILE; i += EF_THREADS) {
            float4 v;
            if (i < na) {
                const int at = a0 + i;
                v.x = frame_atom_coord(__ldg(a.ax128 + at), X0);
                v.y = frame_atom_coord(__ldg(a.ay128 + at), Y0);
                v.z = frame_atom_coord(__ldg(a.az128 + at), Z0);
                v.w = __ldg(a.qw + at);
            } else {
                v = make_float4(1.0e6f, 1.0e6f, 1.0e6f, 0.f);  // far, zero weight
            }
            s_atom[i] = v;
        }
        __syncthreads();
        if (!warp_in) continue;
        float2 acc[NJ];
#pragma unroll
        for (int j = 0; j < NJ; j++) acc[j] = make_float2(0.f, 0.f);
        if (MODE == FAR_TAB_CONST) {
            const float2 fT0 = make_float2(FAR_T0, FAR_T0);
#pragma unroll 2
            for (int i = 0; i < na; i++) {
                const float4 A = s_atom[i];
                const float2 dyz = __fadd2_rn(make_float2(A.y, A.z), npyz);
                const float s = __fmaf_rn(dyz.x, dyz.x, __fmaf_rn(dyz.y, dyz.y, TINY_T2));
                const float2 s2 = make_float2(s, s);
                const float2 ax2 = make_float2(A.x, A.x);
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
                    const float2 dyz = __fadd2_rn(make_float2(A.y, A.z), npyz);
                    const float s = __fmaf_rn(dyz.x, dyz.x, __fmaf_rn(dyz.y, dyz.y, TINY_T2));
                    const float2 s2 = make_float2(s, s);
                    const float2 ax2 = make_float2(A.x, A.x);
                    const float2 q2 = make_float2(A.w, A.w);
                    bool edge = false;
#pragma unroll
                    for (int j = 0; j < NJ; j++) {
                        const float2 dx = __fadd2_rn(ax2, npx[j]);
                        const float2 t2 = __ffma2_rn(dx, dx, s2);
                        const float2 rs = make_float2(rsqrt_approx(t2.x), rsqrt_approx(t2.y));
                        float2 t = __fmul2_rn(t2, rs);
                        t = make_float2(fminf(t.x, tmax.x), fminf(t.y, tmax.y));
                        float2 lo, hi;
                        far_guard_bins(t, lom, him, lo, hi);
                        edge |= (__float_as_uint(lo.x) != __float_as_uint(hi.x)) |
                                (__float_as_uint(lo.y) != __float_as_uint(hi.y));
                        const float T0 = lds_f32(tab_base + (__float_as_uint(lo.x) << 2));
                        const float T1 = lds_f32(tab_base + (__float_as_uint(lo.y) << 2));
                        const float2 wv = __fmul2_rn(q2, rs);
                        acc[j] = __ffma2_rn(wv, make_float2(T0, T1), acc[j]);
                    }
                    hist = (hist << 1) | (edge ? 1u : 0u);
                }
                s_hist[(ib >> 5) * EF_THREADS + tid] = hist << (32 - nb);  // atom ib + k at bit 31 - k
            }
        }
#pragma unroll
        for (int j = 0; j < NJ; j++) tot[j] = __fadd2_rn(tot[j], acc[j]);
        if (MODE != FAR_TAB_CONST && oy + ty < a.n1y && oz + tz < a.n1z) {
            // the flagged atoms of this tile, in atom order (s_hist and s_atom
            // are this tile's); points past the box are not written, not fixed
            const int iy = oy + ty, iz = oz + tz;
            for (int ib = 0; ib < na; ib += 32) {
                uint32_t h = s_hist[(ib >> 5) * EF_THREADS + tid];
                while (h) {
                    const int k = __clz(h);
                    h &= ~(0x80000000u >> k);
                    far_fix_atom<MODE, NJ>(a, s_atom[ib + k], a0 + ib + k, npx, npyz, lom, him, tab_base, ox, iy, iz,
                                           tx, tot, s_cnt);
                }
            }
        }
    }

    const int iy = oy + ty, iz = oz + tz;
    if (iy < a.n1y && iz < a.n1z) {
        float *out = a.partial + (size_t)chunk * (size_t)a.P + ((size_t)iz * a.n1y + iy) * (size_t)a.n1x;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int ix0 = ox + tx + 8 * j, ix1 = ix0 + 4;
            if (ix0 < a.n1x) out[ix0] = tot[j].x;
            if (ix1 < a.n1x) out[ix1] = tot[j].y;
        }
    }
    if (MODE != FAR_TAB_CONST) {
        __syncthreads();
        if (tid < 3) {
            const unsigned v = s_cnt[tid];
            if (v && a.edge_counters) atomicAdd(a.edge_counters + tid, (unsigned long long)v);
            s_cnt[tid] = 0u;
        }
    }
}

// The unit with as many x pairs as the frame has columns inside the box
// (CTA-uniform: only a box's last x frame can be partial).
template <int TILE, int MODE>
__device__ __forceinline__ void far_unit(const FarArgs &a, int f, int chunk, const float4 *s_tab4, float4 *s_atom,
                                         uint32_t *s_hist, unsigned *s_cnt)
{
    static_assert(EF_PAIRS == 4, "x-pair dispatch below");
    const int nj = (a.n1x - (f % a.nfx) * FRAME_X + 7) / 8;
    if (nj >= 4) far_unit_n<TILE, MODE, 4>(a, f, chunk, s_tab4, s_atom, s_hist, s_cnt);
    else if (nj == 3) far_unit_n<TILE, MODE, 3>(a, f, chunk, s_tab4, s_atom, s_hist, s_cnt);
    else if (nj == 2) far_unit_n<TILE, MODE, 2>(a, f, chunk, s_tab4, s_atom, s_hist, s_cnt);
    else far_unit_n<TILE, MODE, 1>(a, f, chunk, s_tab4, s_atom, s_hist, s_cnt);
}

// The unit for the instance's table mode (batch kernel).
template <int TILE>
__device__ __forceinline__ void far_dispatch(const FarArgs &a, int f, int chunk, const float4 *s_tab4, float4 *s_atom,
                                             uint32_t *s_hist, unsigned *s_cnt)
{
    if (a.tab_mode == FAR_TAB_CONST) far_unit<TILE, FAR_TAB_CONST>(a, f, chunk, s_tab4, s_atom, s_hist, s_cnt);
    else far_unit<TILE, FAR_TAB_TABLE>(a, f, chunk, s_tab4, s_atom, s_hist, s_cnt);
}

// Dynamic shared memory of the far kernels: the table (AG_NDIEL floats), the
// atom tile (TILE float4) and the per-thread edge bits (TILE/32 words per thread).
template <int TILE>
__device__ __forceinline__ uint32_t *far_hist_smem(float4 *smem)
{
    return (uint32_t *)(smem + AG_NDIEL / 4 + TILE);
}

// Single instance: one CTA per (frame, chunk) = (blockIdx.x, blockIdx.y).  The
// x-pair count of the box's last x frame (NJ_LAST) is fixed per launch, so a
// grid whose last x frame is full compiles to the full-frame unit alone.
template <int TILE, int NJ_LAST>
__global__ void __launch_bounds__(EF_THREADS, 3) k_emap_far(FarArgs a)
{
    extern __shared__ float4 ef_smem[];
    float4 *s_tab4 = ef_smem;                 // AG_NDIEL floats
    float4 *s_atom = ef_smem + AG_NDIEL / 4;  // TILE entries
    uint32_t *s_hist = far_hist_smem<TILE>(ef_smem);
    __shared__ unsigned s_cnt[3];
    if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0u;
    if (a.tab_mode != FAR_TAB_CONST) load_far_table(s_tab4, a.far_tab);
    __syncthreads();
    const int f = a.frame0 + blockIdx.x;
    const bool last = NJ_LAST < EF_PAIRS && f % a.nfx == a.nfx - 1;
    if (a.tab_mode == FAR_TAB_CONST) {
        if (last) far_unit_n<TILE, FAR_TAB_CONST, NJ_LAST>(a, f, blockIdx.y, s_tab4, s_atom, s_hist, s_cnt);
        else far_unit_n<TILE, FAR_TAB_CONST, EF_PAIRS>(a, f, blockIdx.y, s_tab4, s_atom, s_hist, s_cnt);
    } else {
        if (last) far_unit_n<TILE, FAR_TAB_TABLE, NJ_LAST>(a, f, blockIdx.y, s_tab4, s_atom, s_hist, s_cnt);
        else far_unit_n<TILE, FAR_TAB_TABLE, EF_PAIRS>(a, f, blockIdx.y, s_tab4, s_atom, s_hist, s_cnt);
    }
}

// Many instances, persistent: each CTA takes (instance, frame, chunk) units
// from an atomic counter until none is left; units are numbered instance by
// instance (instances ordered by decreasing work) and never wait on each other.
template <int TILE>
__global__ void __launch_bounds__(EF_THREADS, 3)
k_emap_far_batch(const FarArgs *__restrict__ insts, const long long *__restrict__ unit_begin, int n_inst,
                 unsigned long long *__restrict__ counter)
{
    extern __shared__ float4 ef_smem[];
    float4 *s_tab4 = ef_smem;
    float4 *s_atom = ef_smem + AG_NDIEL / 4;
    uint32_t *s_hist = far_hist_smem<TILE>(ef_smem);
    __shared__ unsigned s_cnt[3];
    if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0u;
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
            if (s_a.tab_mode != FAR_TAB_CONST) load_far_table(s_tab4, s_a.far_tab);
            cur = lo;
        }
        const long long lu = u - unit_begin[lo];
        const int frames = s_a.nfx * s_a.nfy * s_a.nfz;
        const int fr = (int)(lu % frames), ch = (int)(lu / frames);
        far_dispatch<TILE>(s_a, fr, ch, s_tab4, s_atom, s_hist, s_cnt);
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

size_t far_smem_bytes(int tile)
{
    return AG_NDIEL * sizeof(float) + (size_t)tile * sizeof(float4) + (size_t)(tile / 32) * EF_THREADS * sizeof(uint32_t);
}

// Frame z-rows [fz0, fz1) of one instance (fz1 < 0: through the last).
cudaError_t launch_emap_far(const FarArgs &args, int n_chunks, int tile, cudaStream_t s, int fz0, int fz1)
{
    if (tile != 512) return cudaErrorInvalidValue;  // the single-instance kernel stages 512-atom tiles
    FarArgs a = args;
    if (fz1 < 0 || fz1 > a.nfz) fz1 = a.nfz;
    if (fz0 >= fz1) return cudaSuccess;
    a.frame0 = fz0 * a.nfx * a.nfy;
    dim3 grid((unsigned)(a.nfx * a.nfy * (fz1 - fz0)), (unsigned)n_chunks);
    const size_t smem = far_smem_bytes(512);
    const int nj_last = (a.n1x - (a.nfx - 1) * FRAME_X + 7) / 8;  // x pairs of the last frame inside the box
    if (nj_last >= 4) k_emap_far<512, 4><<<grid, EF_THREADS, smem, s>>>(a);
    else if (nj_last == 3) k_emap_far<512, 3><<<grid, EF_THREADS, smem, s>>>(a);
    else if (nj_last == 2) k_emap_far<512, 2><<<grid, EF_THREADS, smem, s>>>(a);
    else k_emap_far<512, 1><<<grid, EF_THREADS, smem, s>>>(a);
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
    const int s512 = (int)far_smem_bytes(512);
    const void *single[] = {(const void *)k_emap_far<512, 1>, (const void *)k_emap_far<512, 2>,
                            (const void *)k_emap_far<512, 3>, (const void *)k_emap_far<512, 4>};
    for (const void *fn : single) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, s512);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e;
    if ((e = cudaFuncSetAttribute((const void *)k_emap_far_batch<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)far_smem_bytes(256))) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute((const void *)k_emap_far_batch<512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  s512)) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute((const void *)k_emap_far_batch<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)far_smem_bytes(1024));
}

// The persistent batch kernel: as many CTAs as fit (at most ctas_per_sm) on
// every SM.  Its shared-memory limit is set by prepare_far_kernels().
template <int TILE>
static cudaError_t far_batch_t(const FarArgs *insts, const long long *unit_begin, int n_inst,
                               unsigned long long *counter, int ctas_per_sm, cudaStream_t s)
{
    const size_t smem = far_smem_bytes(TILE);
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_emap_far_batch<TILE>, EF_THREADS, smem);
    if (e != cudaSuccess) return e;
    const int per_sm = std::max(1, std::min(ctas_per_sm, occ));
    k_emap_far_batch<TILE><<<current_device_sms() * per_sm, EF_THREADS, smem, s>>>(insts, unit_begin, n_inst, counter);
    return cudaGetLastError();
}

cudaError_t launch_emap_far_batch(const FarArgs *insts, const long long *unit_begin, int n_inst,
                                  unsigned long long *counter, int tile, int ctas_per_sm, cudaStream_t s)
{
    if (tile == 256) return far_batch_t<256>(insts, unit_begin, n_inst, counter, ctas_per_sm, s);
    if (tile == 1024) return far_batch_t<1024>(insts, unit_begin, n_inst, counter, ctas_per_sm, s);
    return far_batch_t<512>(insts, unit_begin, n_inst, counter, ctas_per_sm, s);
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
