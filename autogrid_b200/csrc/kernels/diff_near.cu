// Differentiable mode, short-range maps: LOOP 2 of main.cpp:3017-3431 with
// linearly interpolated tables and the 8 A switch (kernels/diff.h), and its
// adjoint.
//   k_closest_h         closest DS/D1 atom of each point, FP64, the reference's
//                       scan (main.cpp:2986-3015: file order, strict <)
//   k_near_lin<R>       forward: a brick of 8x8x4 points per block, one point per
//                       thread; candidate atoms of the cells within 8.05 A of the
//                       brick staged through shared memory; records for each
//                       H-bond min/max slot the atoms attaining the min and max
//   k_near_lin_adj<R>   adjoint: same bricks and staging, pair terms recomputed;
//                       per candidate the 32 points of a warp are reduced with
//                       shuffles and one lane adds the atom's gradient (FP64
//                       atomics); the Hramp gradient on the closest hydrogen's
//                       bond vector is added per point.
#include "agb_device.cuh"
#include "diff.h"
#include "diff_pair.cuh"

namespace agb {

using namespace dfm;

namespace {

constexpr int DF_MAXCELLS = 512;

constexpr int DF_WARPS = DF_THREADS / 32;

template <class R> struct NearLinSmem {
    Atom<R> at[DF_STAGE];
    int ok[DF_MAXCELLS];
    int cells[DF_MAXCELLS], off[DF_MAXCELLS + 1];
    int ncell, total;
    unsigned short wl[DF_WARPS][DF_STAGE];  // per warp: staged slots near its points
    R wbox[DF_WARPS][6];                    // per warp: its points' box (lo xyz, hi xyz), A
};

struct Brick {
    int ix0, iy0, iz0;
    int ix, iy, iz;
    int conf;
    bool valid;
    long long lin;
};

// blockIdx.z runs over (z bricks) x (conformers)
__device__ __forceinline__ Brick brick_of(const DiffArgs &a)
{
    Brick b;
    const int nbz = (a.n1z + DF_BRICK_Z - 1) / DF_BRICK_Z;
    b.conf = blockIdx.z / nbz;
    b.ix0 = blockIdx.x * DF_BRICK_X;
    b.iy0 = blockIdx.y * DF_BRICK_Y;
    b.iz0 = (blockIdx.z % nbz) * DF_BRICK_Z;
    const int t = threadIdx.x;
    b.ix = b.ix0 + t % DF_BRICK_X;
    b.iy = b.iy0 + (t / DF_BRICK_X) % DF_BRICK_Y;
    b.iz = b.iz0 + t / (DF_BRICK_X * DF_BRICK_Y);
    b.valid = b.ix < a.n1x && b.iy < a.n1y && b.iz < a.n1z;
    b.lin = b.valid ? (long long)b.ix + (long long)a.n1x * (b.iy + (long long)a.n1y * b.iz) : 0;
    return b;
}

// This warp's points as a box (lanes outside the grid do not count), kept in
// shared memory for warp_candidates.
template <class R>
__device__ __forceinline__ void warp_box(const Brick &bk, R px, R py, R pz, NearLinSmem<R> &sm)
{
    const R big = (R)3.0e38f;
    R lo[3] = {bk.valid ? px : big, bk.valid ? py : big, bk.valid ? pz : big};
    R hi[3] = {bk.valid ? px : -big, bk.valid ? py : -big, bk.valid ? pz : -big};
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const R a = __shfl_xor_sync(0xffffffffu, lo[d], o), b = __shfl_xor_sync(0xffffffffu, hi[d], o);
            lo[d] = a < lo[d] ? a : lo[d];
            hi[d] = b > hi[d] ? b : hi[d];
        }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int d = 0; d < 3; d++) {
            sm.wbox[w][d] = lo[d];
            sm.wbox[w][3 + d] = hi[d];
        }
    __syncwarp();
}

// Slots j < n of the staged chunk whose atom lies within the cutoff + 0.01 A
// of this warp's box, in staged order (called by all 32 lanes).  Every pair a
// lane of the warp evaluates (r^2 <= 64 in geom) is on the list, so the pairs
// and their order are those of the whole chunk.
template <class R>
__device__ __forceinline__ int warp_candidates(NearLinSmem<R> &sm, int n)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const R *bx = sm.wbox[w];
    const R lim2 = (R)((AG_NBC + 0.01) * (AG_NBC + 0.01));
    int cnt = 0;
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int j = j0 + lane;
        bool keep = false;
        if (j < n) {
            const Atom<R> &at = sm.at[j];
            R e[3];
            const R c[3] = {at.x, at.y, at.z};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const R u = bx[d] - c[d], v = c[d] - bx[3 + d];
                const R m = u > v ? u : v;
                e[d] = m > (R)0 ? m : (R)0;
            }
            keep = e[0] * e[0] + e[1] * e[1] + e[2] * e[2] <= lim2;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) sm.wl[w][cnt + __popc(m & ((1u << lane) - 1u))] = (unsigned short)j;
        cnt += __popc(m);
    }
    __syncwarp();
    return cnt;
}

// Cells whose box lies within DF_RADIUS of the brick's box, in cell order,
// with the running offsets of their atoms.
template <class R>
__device__ void brick_cells(const DiffArgs &a, const ConfView &v, const Brick &bk, NearLinSmem<R> &sm)
{
    const int ix1 = min(bk.ix0 + DF_BRICK_X - 1, a.n1x - 1), iy1 = min(bk.iy0 + DF_BRICK_Y - 1, a.n1y - 1),
              iz1 = min(bk.iz0 + DF_BRICK_Z - 1, a.n1z - 1);
    const double lo[3] = {(bk.ix0 - a.nex) * a.spacing, (bk.iy0 - a.ney) * a.spacing, (bk.iz0 - a.nez) * a.spacing};
    const double hi[3] = {(ix1 - a.nex) * a.spacing, (iy1 - a.ney) * a.spacing, (iz1 - a.nez) * a.spacing};
    const int nc[3] = {a.ncx, a.ncy, a.ncz};
    int c0[3], c1[3];
    bool empty = false;
    for (int i = 0; i < 3; i++) {
        c0[i] = (int)floor((lo[i] - DF_RADIUS - a.cell0[i]) / a.cell_size);
        c1[i] = (int)floor((hi[i] + DF_RADIUS - a.cell0[i]) / a.cell_size);
        c0[i] = max(c0[i], 0);
        c1[i] = min(c1[i], nc[i] - 1);
        if (c0[i] > c1[i]) empty = true;
    }
    const int wx = c1[0] - c0[0] + 1, wy = c1[1] - c0[1] + 1, wz = c1[2] - c0[2] + 1;
    const int n = empty ? 0 : min(wx * wy * wz, DF_MAXCELLS);
    for (int k = threadIdx.x; k < n; k += DF_THREADS) {
        const int cx = c0[0] + k % wx, cy = c0[1] + (k / wx) % wy, cz = c0[2] + k / (wx * wy);
        const int cc[3] = {cx, cy, cz};
        double d2 = 0.0;
        for (int i = 0; i < 3; i++) {
            const double blo = a.cell0[i] + cc[i] * a.cell_size, bhi = blo + a.cell_size;
            const double g = fmax(fmax(blo - hi[i], lo[i] - bhi), 0.0);
            d2 += g * g;
        }
        const int cid = cx + a.ncx * (cy + a.ncy * cz);
        const int cnt = v.cell_start[cid + 1] - v.cell_start[cid];
        sm.ok[k] = (d2 <= DF_RADIUS * DF_RADIUS && cnt > 0) ? cid : -1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int m = 0, tot = 0;
        for (int k = 0; k < n; k++) {
            const int cid = sm.ok[k];
            if (cid < 0) continue;
            sm.cells[m] = cid;
            sm.off[m] = tot;
            tot += v.cell_start[cid + 1] - v.cell_start[cid];
            m++;
        }
        sm.off[m] = tot;
        sm.ncell = m;
        sm.total = tot;
    }
    __syncthreads();
}

// Stage candidates [c0, c0 + DF_STAGE) of the brick into shared memory.
template <class R>
__device__ void stage_chunk(const DiffArgs &a, const ConfView &v, NearLinSmem<R> &sm, int c0)
{
    const int k = c0 + threadIdx.x;
    if (threadIdx.x < DF_STAGE && k < sm.total) {
        int lo = 0, hi = sm.ncell - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sm.off[mid] <= k) lo = mid;
            else hi = mid - 1;
        }
        const int ia = v.cell_atoms[v.cell_start[sm.cells[lo]] + (k - sm.off[lo])];
        Atom<R> &t = sm.at[threadIdx.x];
        t.x = (R)v.x[ia]; t.y = (R)v.y[ia]; t.z = (R)v.z[ia];
        t.q = (R)v.q[ia]; t.vol = (R)a.vol[ia]; t.solpar = (R)a.solpar[ia];
        for (int i = 0; i < 3; i++) {
            t.rv[i] = (R)v.rv[3 * ia + i];
            t.rv2[i] = (R)v.rv2[3 * ia + i];
        }
        t.meta = a.meta[ia];
        t.idx = ia;
    }
}

template <class R> __device__ __forceinline__ R covalent_value(const DiffArgs &a, R px, R py, R pz)
{
    // main.cpp:2866-2879
    const R d0 = (R)a.cov_pos[0] - px, d1 = (R)a.cov_pos[1] - py, d2 = (R)a.cov_pos[2] - pz;
    R rc = sqrt_(d0 * d0 + d1 * d1 + d2 * d2) / (R)a.cov_half_width;
    if (rc < (R)DF_TINY) rc = (R)DF_TINY;
    return (R)a.cov_barrier * ((R)1 - exp_((R)-0.69314718055994531 * rc * rc));
}

// MS slots and MM min/max registers per point: the general instantiation
// holds DF_MAXS / DF_MAXMM; map sets of at most DF_LEAN_S slots without
// H-bond min/max (Vina maps, plain AD4 subsets) take the lean one, whose
// registers leave room for 3 resident CTAs per SM.  ANG = false: no slot uses
// the directional factors (DiffArgs::need_ang), so none are evaluated; the
// lean angle-free kernels fit 64 registers and run 4 CTAs per SM.
template <class R, int MS, int MM, int MINB, bool ANG = true>
__global__ void __launch_bounds__(DF_THREADS, MINB)
k_near_lin(DiffArgs a, const R2<R> *__restrict__ vdw, const R2<R> *__restrict__ sol, R *__restrict__ maps,
           const int *__restrict__ chs, int *__restrict__ mmarg)
{
    constexpr int MMA = MM > 0 ? MM : 1;
    __shared__ NearLinSmem<R> sm;
    const Brick bk = brick_of(a);
    const ConfView v = conf_view(a, DiffGrads{}, bk.conf);
    chs += bk.conf * a.P;
    maps += (long long)bk.conf * a.n_maps_out * a.P;
    mmarg += 2LL * bk.conf * a.n_mm * a.P;
    const R px = (R)((bk.ix - a.nex) * a.spacing), py = (R)((bk.iy - a.ney) * a.spacing),
            pz = (R)((bk.iz - a.nez) * a.spacing);
    const int ch = bk.valid ? chs[bk.lin] : -1;
    R rvh[3] = {0, 0, 0};
    if (ch >= 0)
        for (int i = 0; i < 3; i++) rvh[i] = (R)v.rv[3 * ch + i];
    R E[MS], hmin[MMA], hmax[MMA];
    int amin[MMA], amax[MMA];
#pragma unroll
    for (int s = 0; s < MS; s++) E[s] = 0;
#pragma unroll
    for (int s = 0; s < MMA; s++) { hmin[s] = (R)999999.; hmax[s] = (R)-999999.; amin[s] = -1; amax[s] = -1; }

    brick_cells(a, v, bk, sm);
    warp_box(bk, px, py, pz, sm);
    for (int c0 = 0; c0 < sm.total; c0 += DF_STAGE) {
        __syncthreads();
        stage_chunk(a, v, sm, c0);
        __syncthreads();
        const int n = min(DF_STAGE, sm.total - c0);
        const int cnt = warp_candidates(sm, n);
        if (!bk.valid) continue;
        const unsigned short *wl = sm.wl[threadIdx.x >> 5];
        for (int k = 0; k < cnt; k++) {
            const Atom<R> at = sm.at[wl[k]];
            Geom<R> g;
            if (!geom(a.need_sol ? sol : nullptr, at, px, py, pz, g)) continue;
            Ang<R> an;
            if (ANG)
                angular((at.meta >> DM_HB_SHIFT) & 7, (at.meta >> DM_REXP_SHIFT) & 7, (at.meta & DM_DIS) != 0,
                        ch >= 0 && at.idx != ch, g.dn, at.rv, at.rv2, rvh, an);
            else
                ang_plain(an);
            pair_fwd<R, MS, MM>(a, vdw, g, at, an, E, hmin, hmax, amin, amax);
        }
    }
    if (!bk.valid) return;
#pragma unroll
    for (int s = 0; s < MS; s++) {
        if (s >= a.n_slots) break;
        R v = E[s];
        if (s < MM && s < a.n_mm) {
            // H-bond finaliser, main.cpp:3420-3431
            if (amin[s] >= 0) v += hmin[s] + (hmax[s] > (R)0 ? hmax[s] : (R)0);
            mmarg[(2LL * s) * a.P + bk.lin] = amin[s];
            mmarg[(2LL * s + 1) * a.P + bk.lin] = hmax[s] > (R)0 ? amax[s] : -1;
        }
        if (a.slot_kind[s] == DK_COV) v += covalent_value<R>(a, px, py, pz);
        maps[(long long)a.slot_map[s] * a.P + bk.lin] = v;
    }
}

template <class R> __device__ __forceinline__ R warp_sum(R v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class R, int MS, int MM, int MINB, bool ANG = true>
__global__ void __launch_bounds__(DF_THREADS, MINB)
k_near_lin_adj(DiffArgs a, const R2<R> *__restrict__ vdw, const R2<R> *__restrict__ sol,
               const R *__restrict__ g_maps, const int *__restrict__ chs, const int *__restrict__ mmarg,
               DiffGrads gr_all)
{
    constexpr int MMA = MM > 0 ? MM : 1;
    __shared__ NearLinSmem<R> sm;
    const Brick bk = brick_of(a);
    const ConfView v = conf_view(a, gr_all, bk.conf);
    const DiffGrads gr = v.g;
    chs += bk.conf * a.P;
    g_maps += (long long)bk.conf * a.n_maps_out * a.P;
    mmarg += 2LL * bk.conf * a.n_mm * a.P;
    const R px = (R)((bk.ix - a.nex) * a.spacing), py = (R)((bk.iy - a.ney) * a.spacing),
            pz = (R)((bk.iz - a.nez) * a.spacing);
    const int ch = bk.valid ? chs[bk.lin] : -1;
    R rvh[3] = {0, 0, 0}, g_rvh[3] = {0, 0, 0};
    if (ch >= 0)
        for (int i = 0; i < 3; i++) rvh[i] = (R)v.rv[3 * ch + i];
    R gs[MS];
    int amin[MMA], amax[MMA];
#pragma unroll
    for (int s = 0; s < MS; s++)
        gs[s] = (bk.valid && s < a.n_slots) ? g_maps[(long long)a.slot_map[s] * a.P + bk.lin] : (R)0;
#pragma unroll
    for (int s = 0; s < MMA; s++) {
        const bool has = bk.valid && s < MM && s < a.n_mm;
        amin[s] = has ? mmarg[(2LL * s) * a.P + bk.lin] : -1;
        amax[s] = has ? mmarg[(2LL * s + 1) * a.P + bk.lin] : -1;
    }
    const int lane = threadIdx.x & 31;

    brick_cells(a, v, bk, sm);
    warp_box(bk, px, py, pz, sm);
    for (int c0 = 0; c0 < sm.total; c0 += DF_STAGE) {
        __syncthreads();
        stage_chunk(a, v, sm, c0);
        __syncthreads();
        const int n = min(DF_STAGE, sm.total - c0);
        const int cnt = warp_candidates(sm, n);
        const unsigned short *wl = sm.wl[threadIdx.x >> 5];
        for (int k = 0; k < cnt; k++) {
            const Atom<R> at = sm.at[wl[k]];
            Geom<R> g;
            const bool in = bk.valid && geom(a.need_sol ? sol : nullptr, at, px, py, pz, g);
            if (!__any_sync(0xffffffffu, in)) continue;
            const int hb = (at.meta >> DM_HB_SHIFT) & 7;
            const bool dis = (at.meta & DM_DIS) != 0;
            R g_d[3] = {0, 0, 0}, g_rv[3] = {0, 0, 0}, g_rv2[3] = {0, 0, 0}, G_q = 0;
            if (in) {
                Ang<R> an;
                if (ANG)
                    angular(hb, (at.meta >> DM_REXP_SHIFT) & 7, dis, ch >= 0 && at.idx != ch, g.dn, at.rv, at.rv2,
                            rvh, an);
                else
                    ang_plain(an);
                R G_x = 0, G_racc = 0, G_rdon = 0, G_H = 0;
                pair_bwd<R, MS, MM>(a, vdw, g, at, an, gs, amin, amax, G_x, G_racc, G_rdon, G_H, G_q);
                R g_dn[3] = {0, 0, 0};
                if (ANG)
                    angular_bwd(hb, dis, an, G_racc, G_rdon, G_H, g.dn, at.rv, at.rv2, rvh, g_dn, g_rv, g_rv2,
                                g_rvh);
                geom_bwd(g, G_x, g_dn, g_d);
            }
            // the candidate is the same for the whole warp: reduce, one lane adds
            // G_q comes from desolvation terms only
            const R sx = warp_sum(g_d[0]), sy = warp_sum(g_d[1]), sz = warp_sum(g_d[2]);
            const R sq = a.need_sol ? warp_sum(G_q) : (R)0;
            R sr[3] = {0, 0, 0}, sr2[3] = {0, 0, 0};
            const bool has_rv = ANG && (hb == 2 || hb == 4 || hb == 5);
            const bool has_rv2 = ANG && hb == 5 && !dis;
            if (has_rv)
                for (int i = 0; i < 3; i++) sr[i] = warp_sum(g_rv[i]);
            if (has_rv2)
                for (int i = 0; i < 3; i++) sr2[i] = warp_sum(g_rv2[i]);
            if (lane == 0) {
                const long long ia = at.idx;
                atomicAdd(gr.xyz + 3 * ia, (double)sx);
                atomicAdd(gr.xyz + 3 * ia + 1, (double)sy);
                atomicAdd(gr.xyz + 3 * ia + 2, (double)sz);
                if (sq != (R)0) atomicAdd(gr.q + ia, (double)sq);
                if (has_rv)
                    for (int i = 0; i < 3; i++) atomicAdd(gr.rv + 3 * ia + i, (double)sr[i]);
                if (has_rv2)
                    for (int i = 0; i < 3; i++) atomicAdd(gr.rv2 + 3 * ia + i, (double)sr2[i]);
            }
        }
    }
    if (ch >= 0 && (g_rvh[0] != (R)0 || g_rvh[1] != (R)0 || g_rvh[2] != (R)0))
        for (int i = 0; i < 3; i++) atomicAdd(gr.rv + 3LL * ch + i, (double)g_rvh[i]);
}

constexpr int CH_THREADS = 256;

__global__ void __launch_bounds__(CH_THREADS) k_closest_h(DiffArgs a, int *__restrict__ ch)
{
    __shared__ double sx[CH_THREADS], sy[CH_THREADS], sz[CH_THREADS];
    __shared__ int sidx[CH_THREADS];
    const ConfView v = conf_view(a, DiffGrads{}, blockIdx.y);
    ch += blockIdx.y * a.P;
    const long long lin = (long long)blockIdx.x * CH_THREADS + threadIdx.x;
    const bool valid = lin < a.P;
    const long long l = valid ? lin : 0;
    const int ix = (int)(l % a.n1x), iy = (int)((l / a.n1x) % a.n1y), iz = (int)(l / ((long long)a.n1x * a.n1y));
    const double cx = (double)(ix - a.nex) * a.spacing, cy = (double)(iy - a.ney) * a.spacing,
                 cz = (double)(iz - a.nez) * a.spacing;
    // The reference keeps the first H atom in file order with the strictly
    // smallest r = sqrt(d0^2 + d1^2 + d2^2).  sqrt is monotonic, so only a
    // strictly smaller square can give a strictly smaller r; when the squares
    // differ by more than 2^-48 relative, the correctly rounded roots differ
    // too, and only closer squares need the roots themselves compared.
    double best2 = 999999. * 999999.;  // rmin = 999999, exactly
    int best = -1;
    for (int h0 = 0; h0 < a.n_h; h0 += CH_THREADS) {
        const int nh = min(CH_THREADS, a.n_h - h0);
        __syncthreads();
        if (threadIdx.x < nh) {
            const int ia = a.h_index[h0 + threadIdx.x];
            sx[threadIdx.x] = v.x[ia]; sy[threadIdx.x] = v.y[ia]; sz[threadIdx.x] = v.z[ia];
            sidx[threadIdx.x] = ia;
        }
        __syncthreads();
        for (int j = 0; j < nh; j++) {
            const double d0 = __dsub_rn(sx[j], cx), d1 = __dsub_rn(sy[j], cy), d2 = __dsub_rn(sz[j], cz);
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
            if (r2 < best2 &&
                (best2 - r2 > best2 * 3.552713678800501e-15 /* 2^-48 */ || __dsqrt_rn(r2) < __dsqrt_rn(best2))) {
                best2 = r2;
                best = sidx[j];
            }
        }
    }
    if (valid) ch[lin] = best;
}

dim3 brick_grid(const DiffArgs &a)
{
    return dim3((unsigned)((a.n1x + DF_BRICK_X - 1) / DF_BRICK_X), (unsigned)((a.n1y + DF_BRICK_Y - 1) / DF_BRICK_Y),
                (unsigned)((a.n1z + DF_BRICK_Z - 1) / DF_BRICK_Z * a.n_conf));
}

}  // namespace

cudaError_t launch_closest_h(const DiffArgs &a, int *ch, cudaStream_t s)
{
    if (a.P == 0) return cudaSuccess;
    k_closest_h<<<dim3((unsigned)((a.P + CH_THREADS - 1) / CH_THREADS), (unsigned)a.n_conf), CH_THREADS, 0, s>>>(a, ch);
    return cudaGetLastError();
}

cudaError_t launch_near_lin(bool fp64, const DiffArgs &a, const void *vdw, const void *sol, void *maps,
                            const int *ch, int *mmarg, cudaStream_t s)
{
    if (a.P == 0 || a.n_slots == 0) return cudaSuccess;
    const bool lean = a.n_slots <= DF_LEAN_S && a.n_mm == 0;
    const bool mid = a.n_slots <= DF_LEAN_S && a.n_mm <= DF_MID_MM;
    if (fp64)
        k_near_lin<double, DF_MAXS, DF_MAXMM, 1><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<double> *)vdw, (const R2<double> *)sol, (double *)maps, ch, mmarg);
    else if (lean && !a.need_ang)
        k_near_lin<float, DF_LEAN_S, 0, 4, false><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (float *)maps, ch, mmarg);
    else if (mid && !lean)
        k_near_lin<float, DF_LEAN_S, DF_MID_MM, 3><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (float *)maps, ch, mmarg);
    else if (lean)
        k_near_lin<float, DF_LEAN_S, 0, 3><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (float *)maps, ch, mmarg);
    else
        k_near_lin<float, DF_MAXS, DF_MAXMM, 2><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (float *)maps, ch, mmarg);
    return cudaGetLastError();
}

cudaError_t launch_near_lin_adj(bool fp64, const DiffArgs &a, const void *vdw, const void *sol, const void *g_maps,
                                const int *ch, const int *mmarg, DiffGrads g, cudaStream_t s)
{
    if (a.P == 0 || a.n_slots == 0) return cudaSuccess;
    const bool lean = a.n_slots <= DF_LEAN_S && a.n_mm == 0;
    const bool mid = a.n_slots <= DF_LEAN_S && a.n_mm <= DF_MID_MM;
    if (fp64)
        k_near_lin_adj<double, DF_MAXS, DF_MAXMM, 1><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<double> *)vdw, (const R2<double> *)sol, (const double *)g_maps, ch, mmarg, g);
    else if (lean && !a.need_ang)
        k_near_lin_adj<float, DF_LEAN_S, 0, 4, false><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (const float *)g_maps, ch, mmarg, g);
    else if (mid && !lean)
        k_near_lin_adj<float, DF_LEAN_S, DF_MID_MM, 3><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (const float *)g_maps, ch, mmarg, g);
    else if (lean)
        k_near_lin_adj<float, DF_LEAN_S, 0, 3><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (const float *)g_maps, ch, mmarg, g);
    else
        k_near_lin_adj<float, DF_MAXS, DF_MAXMM, 2><<<brick_grid(a), DF_THREADS, 0, s>>>(
            a, (const R2<float> *)vdw, (const R2<float> *)sol, (const float *)g_maps, ch, mmarg, g);
    return cudaGetLastError();
}

}  // namespace agb
