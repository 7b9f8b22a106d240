// C ABI of the differentiable mode (kernels/diff.h defines it): problem
// binding, cell list, interpolation tables, forward and adjoint launches.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "autogrid_b200.h"
#include "kernels/diff.h"
#include "kernels/kernels.h"

namespace agb {
void set_last_error(const std::string &m);
ag_status validate_problem(const ag_problem *p);
ag_status validate_problem_box(const ag_problem *p);
cudaStream_t context_stream(const ag_context *c);
int context_device(const ag_context *c);
bool device_accessible(const void *ptr, int device);
}  // namespace agb

using namespace agb;

namespace {

ag_status fail_cuda(cudaError_t e, const char *what)
{
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return AG_ERR_CUDA;
}

#define DF_CK(call)                                        \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call); \
    } while (0)

// What the atom term of atom map m does for a receptor atom of class hb and
// disorder flag dis: the branch conditions of main.cpp:3290-3379.
uint8_t action_of(const ag_problem *p, int m, int hb, int dis)
{
    if (!p->map_is_hbonder[m]) return DA_PLAIN;
    const int mh = p->map_hbond[m];
    const bool rec_donor = hb == 1 || hb == 2 || hb == 6;
    if ((mh == 3 || mh == 5 || mh == 6) && rec_donor) return dis ? DA_SUMA_DIS : DA_SUMA;
    if ((mh == 4 || mh == 6) && rec_donor) return DA_MMA;
    if ((mh == 1 || mh == 2 || mh == 6) && (hb > 2 || hb == 6)) return dis ? DA_SUMD_DIS : DA_MMD;
    return DA_PLAIN;
}

struct Slot {
    int map = -1, kind = DK_ATOM, tab = -1, desolv = 0;
    bool mm = false;
    uint8_t act[16] = {};
};

}  // namespace

struct ag_diff {
    ag_context *ctx = nullptr;
    cudaStream_t stream = nullptr;
    int device = 0;
    bool fp64 = false;
    size_t esz = 4;
    int N = 0, n_conf = 1, n_maps = 0, n_atom_maps = 0, elec = -1;
    // distance maps after the energy maps (main.cpp:2958-2966): n_out maps per conformer
    int floating = 0, constriction = 0, n_out = 0;
    double cmap_cutoff = 7.5;
    bool need_h = false;
    long long P = 0;
    size_t ncells = 0;
    std::vector<double> coord, charge, rv, rv2;  // [conf][...]
    std::vector<int> h_index;
    DiffArgs args{};
    // device
    std::vector<void *> allocs;
    double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr, *d_q = nullptr, *d_vol = nullptr, *d_solpar = nullptr;
    double *d_rv = nullptr, *d_rv2 = nullptr, *d_grad = nullptr;
    int *d_meta = nullptr, *d_h = nullptr, *d_cell_start = nullptr, *d_cell_atoms = nullptr;
    int *d_ch = nullptr, *d_mmarg = nullptr;
    void *d_vdw = nullptr, *d_sol = nullptr, *d_eps = nullptr, *d_maps = nullptr, *d_gmaps = nullptr;
    cudaEvent_t ev[6] = {};
    float fwd_ms = 0, ch_ms = 0, bwd_ms = 0;
    bool have_ch = false, have_fwd = false;
    // device-resident atom updates (ag_diff_set_atoms_device)
    int *d_topo = nullptr, *d_cell_of = nullptr, *d_cell_count = nullptr, *d_bad = nullptr;
    bool host_stale = false;  // the host copies lag the device arrays

    ~ag_diff()
    {
        cudaSetDevice(device);
        for (void *p : allocs) cudaFree(p);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
    }
    template <class T> cudaError_t alloc(T **p, size_t n)
    {
        void *v = nullptr;
        cudaError_t e = cudaMalloc(&v, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) {
            allocs.push_back(v);
            *p = (T *)v;
        }
        return e;
    }
    size_t map_bytes() const { return esz * (size_t)P * n_out * n_conf; }
    DevProblem conformer_geometry(int k) const;
    ag_status upload_conformer(int k);
    ag_status refresh_host();
};

namespace {

// vdW rows [type][bin][stride]: slot s holds the table of its atom map
// (slot_tab[s]; zero for slots without a pair term).
template <class R>
void build_tables(const ag_problem *p, const DiffArgs &A, std::vector<R2<R>> &vdw, std::vector<R2<R>> &sol,
                  std::vector<R2<R>> &eps)
{
    const int nT = p->n_rec_types, nAM = p->n_atom_maps, W = A.tab_stride;
    vdw.assign((size_t)std::max(nT, 1) * AG_NEINT * W, R2<R>{R(0), R(0)});
    for (int t = 0; t < nT; t++)
        for (int s = 0; s < A.n_slots; s++) {
            const int m = A.slot_tab[s];
            if (m < 0) continue;
            const float *src = p->e_vdw_hb + ((size_t)t * nAM + m) * AG_NEINT;
            for (int b = 0; b < AG_NEINT; b++) {
                const double v = src[b], nx = (b < AG_NEINT - 1) ? (double)src[b + 1] : v;
                vdw[((size_t)t * AG_NEINT + b) * W + s] = R2<R>{R(v), R(nx - v)};
            }
        }
    sol.resize(AG_NEINT);
    for (int b = 0; b < AG_NEINT; b++)
        sol[b] = R2<R>{R(p->sol_fn[b]), R(p->sol_fn[b + 1] - p->sol_fn[b])};
    eps.resize(AG_NDIEL);
    auto f = [&](int b) { return p->dddiel ? p->r_epsilon_fn[b] * p->coeff_estat : p->invdielcal * p->coeff_estat; };
    for (int b = 0; b < AG_NDIEL; b++) {
        const double v = f(b), nx = (b < AG_NDIEL - 1) ? f(b + 1) : v;
        eps[b] = R2<R>{R(v), R(nx - v)};
    }
}

template <class R> cudaError_t put(void **dst, const std::vector<R> &v, ag_diff *d)
{
    R *p = nullptr;
    cudaError_t e = d->alloc(&p, v.size());
    if (e != cudaSuccess) return e;
    *dst = p;
    return cudaMemcpy(p, v.data(), v.size() * sizeof(R), cudaMemcpyHostToDevice);
}

bool act_uses_angles(uint8_t a) { return a != DA_PLAIN && a != DA_NONE; }
bool act_uses_ramp(uint8_t a) { return a == DA_SUMA || a == DA_SUMA_DIS || a == DA_SUMD_DIS; }

}  // namespace

// The distance-map kernels' view of conformer k: its atoms and the grid.
DevProblem ag_diff::conformer_geometry(int k) const
{
    DevProblem g;
    std::memset(&g, 0, sizeof g);
    g.n_atoms = N;
    g.n1x = args.n1x; g.n1y = args.n1y; g.n1z = args.n1z;
    g.nex = args.nex; g.ney = args.ney; g.nez = args.nez;
    g.P = P;
    g.spacing = args.spacing;
    g.x = d_x + (size_t)N * k; g.y = d_y + (size_t)N * k; g.z = d_z + (size_t)N * k;
    return g;
}

// Coordinates, charges, bond vectors and cell list of conformer k.
ag_status ag_diff::upload_conformer(int k)
{
    const size_t o1 = (size_t)k * N, o3 = 3 * o1;
    std::vector<double> x(N), y(N), z(N);
    for (int a = 0; a < N; a++) { x[a] = coord[o3 + 3 * a]; y[a] = coord[o3 + 3 * a + 1]; z[a] = coord[o3 + 3 * a + 2]; }
    // cell list over the grid box grown by DF_RADIUS; atoms outside it have no
    // point within the 8 A cutoff
    std::vector<int> cell_of(N, -1), start(ncells + 1, 0);
    const int nc[3] = {args.ncx, args.ncy, args.ncz};
    for (int a = 0; a < N; a++) {
        int c[3];
        bool in = true;
        const double pc[3] = {x[a], y[a], z[a]};
        for (int i = 0; i < 3; i++) {
            const double u = std::floor((pc[i] - args.cell0[i]) / args.cell_size);
            if (!(u >= 0 && u < nc[i])) { in = false; break; }
            c[i] = (int)u;
        }
        if (!in) continue;
        cell_of[a] = c[0] + args.ncx * (c[1] + args.ncy * c[2]);
        start[cell_of[a] + 1]++;
    }
    for (size_t i = 1; i < start.size(); i++) start[i] += start[i - 1];
    std::vector<int> fill(start.begin(), start.end() - 1), atoms(std::max(N, 1), 0);
    for (int a = 0; a < N; a++)
        if (cell_of[a] >= 0) atoms[fill[cell_of[a]]++] = a;
    const size_t nb = (size_t)N * sizeof(double);
    DF_CK(cudaMemcpyAsync(d_x + o1, x.data(), nb, cudaMemcpyHostToDevice, stream));
    DF_CK(cudaMemcpyAsync(d_y + o1, y.data(), nb, cudaMemcpyHostToDevice, stream));
    DF_CK(cudaMemcpyAsync(d_z + o1, z.data(), nb, cudaMemcpyHostToDevice, stream));
    DF_CK(cudaMemcpyAsync(d_q + o1, charge.data() + o1, nb, cudaMemcpyHostToDevice, stream));
    DF_CK(cudaMemcpyAsync(d_rv + o3, rv.data() + o3, 3 * nb, cudaMemcpyHostToDevice, stream));
    DF_CK(cudaMemcpyAsync(d_rv2 + o3, rv2.data() + o3, 3 * nb, cudaMemcpyHostToDevice, stream));
    DF_CK(cudaMemcpyAsync(d_cell_start + (size_t)k * (ncells + 1), start.data(), start.size() * sizeof(int),
                          cudaMemcpyHostToDevice, stream));
    DF_CK(cudaMemcpyAsync(d_cell_atoms + o1, atoms.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice, stream));
    DF_CK(cudaStreamSynchronize(stream));  // host vectors are locals
    return AG_OK;
}

// Host copies of every conformer's coordinates, charges and bond vectors from
// the device arrays (after device-resident updates).
ag_status ag_diff::refresh_host()
{
    if (!host_stale) return AG_OK;
    const size_t NK = (size_t)N * n_conf;
    std::vector<double> x(NK), y(NK), z(NK);
    DF_CK(cudaMemcpyAsync(x.data(), d_x, NK * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DF_CK(cudaMemcpyAsync(y.data(), d_y, NK * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DF_CK(cudaMemcpyAsync(z.data(), d_z, NK * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DF_CK(cudaMemcpyAsync(charge.data(), d_q, NK * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DF_CK(cudaMemcpyAsync(rv.data(), d_rv, 3 * NK * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DF_CK(cudaMemcpyAsync(rv2.data(), d_rv2, 3 * NK * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DF_CK(cudaStreamSynchronize(stream));
    for (size_t i = 0; i < NK; i++) {
        coord[3 * i] = x[i];
        coord[3 * i + 1] = y[i];
        coord[3 * i + 2] = z[i];
    }
    host_stale = false;
    return AG_OK;
}

extern "C" {

ag_status ag_diff_create_batch(ag_context *ctx, const ag_problem *p, const ag_opts *o, int32_t n_conformers,
                               ag_diff **out)
{
    if (!ctx || !p || !o || !out) { set_last_error("ag_diff_create: null argument"); return AG_ERR_INVALID; }
    *out = nullptr;
    if (n_conformers < 1 || n_conformers > 4096) {
        set_last_error("ag_diff_create_batch: n_conformers out of range [1, 4096]");
        return AG_ERR_INVALID;
    }
    if (o->table_mode != AG_TABLE_LINEAR) {
        set_last_error("ag_diff_create: opts->table_mode must be AG_TABLE_LINEAR");
        return AG_ERR_INVALID;
    }
    if (o->precision != AG_PREC_FP32 && o->precision != AG_PREC_FP64) {
        set_last_error("ag_diff_create: unknown precision");
        return AG_ERR_INVALID;
    }
    if (p->report_collisions) {
        set_last_error("ag_diff_create: the differentiable mode does not report collisions (map_receptor_interior off)");
        return AG_ERR_UNSUPPORTED;
    }
    // the closest-hydrogen requirement is checked below, only if a map uses Hramp
    ag_problem pv = *p;
    const int nAM = p->n_atom_maps;
    ag_status st = validate_problem_box(&pv);  // any box: a z-slab of a grid is a shard
    if (st != AG_OK && st != AG_ERR_NO_CLOSEST_H) return st;
    // tables in device memory (ag_tables_build): read them here once; the
    // interpolation pairs are formed on the host at creation
    std::vector<float> h_vdw;
    std::vector<double> h_sol, h_eps;
    {
        cudaPointerAttributes at{};
        const bool dev = cudaPointerGetAttributes(&at, p->e_vdw_hb) == cudaSuccess && at.type == cudaMemoryTypeDevice;
        cudaGetLastError();
        if (dev) {
            DF_CK(cudaSetDevice(context_device(ctx)));
            h_vdw.resize((size_t)std::max(p->n_rec_types, 1) * std::max(nAM, 1) * AG_NEINT);
            h_sol.resize(AG_NDIEL);
            DF_CK(cudaMemcpy(h_vdw.data(), p->e_vdw_hb, (size_t)p->n_rec_types * nAM * AG_NEINT * sizeof(float),
                             cudaMemcpyDeviceToHost));
            DF_CK(cudaMemcpy(h_sol.data(), p->sol_fn, AG_NDIEL * sizeof(double), cudaMemcpyDeviceToHost));
            pv.e_vdw_hb = h_vdw.data();
            pv.sol_fn = h_sol.data();
            if (p->dddiel) {
                h_eps.resize(AG_NDIEL);
                DF_CK(cudaMemcpy(h_eps.data(), p->r_epsilon_fn, AG_NDIEL * sizeof(double), cudaMemcpyDeviceToHost));
                pv.r_epsilon_fn = h_eps.data();
            }
            p = &pv;
        }
    }
    // Slots: every map but the e map.  The atom term of map m and the
    // desolvation target follow the reference's map loop (main.cpp:3286-3390):
    // a covalent map is skipped whole; with separate desolvation maps the
    // desolvation of map m goes to map m+1.
    std::vector<Slot> slots;
    std::vector<int> tab_of(std::max(nAM, 1), -1), desolv_of(std::max(nAM, 1), 0);
    for (int m = 0; m < nAM; m++) {
        if (p->map_is_covalent[m]) continue;
        tab_of[m] = m;
        int dm = m;
        if (p->separate_desolvation_maps) dm = ++m;
        if (dm >= nAM) {
            set_last_error("ag_diff_create: desolvation partner past the last atom map");
            return AG_ERR_INVALID;
        }
        desolv_of[dm] = 1;
    }
    bool need_ang = false, need_h = false;
    for (int m = 0; m < nAM; m++) {
        Slot s;
        s.map = m;
        s.kind = p->map_is_covalent[m] ? DK_COV : DK_ATOM;  // covalent: Gaussian added at the end
        s.tab = tab_of[m];
        // a desolvation term with zero probe parameters adds exactly zero
        s.desolv = desolv_of[m] && (p->map_solpar_probe[m] != 0.0 || p->map_vol_probe[m] != 0.0);
        if (s.tab >= 0)
            for (int dis = 0; dis < 2; dis++)
                for (int hb = 0; hb < 8; hb++) {
                    const uint8_t a = action_of(p, s.tab, hb, dis);
                    s.act[hb + 8 * dis] = a;
                    if (a == DA_MMA || a == DA_MMD) s.mm = true;
                    need_ang |= act_uses_angles(a);
                    need_h |= act_uses_ramp(a);
                }
        slots.push_back(s);
    }
    if (p->dsolv_map >= 0) {
        Slot s;
        s.map = p->dsolv_map;
        s.kind = DK_D;
        slots.push_back(s);
    }
    if (need_h && st == AG_ERR_NO_CLOSEST_H) return st;
    std::stable_partition(slots.begin(), slots.end(), [](const Slot &s) { return s.mm; });
    const int n_mm = (int)std::count_if(slots.begin(), slots.end(), [](const Slot &s) { return s.mm; });
    if ((int)slots.size() > DF_MAXS || n_mm > DF_MAXMM) {
        set_last_error("ag_diff_create: the differentiable mode takes at most 16 maps besides the e map, "
                       "at most 8 with H-bond min/max terms");
        return AG_ERR_UNSUPPORTED;
    }

    cudaError_t ce = cudaSetDevice(context_device(ctx));
    if (ce != cudaSuccess) return fail_cuda(ce, "cudaSetDevice");
    std::unique_ptr<ag_diff> d(new ag_diff());
    d->ctx = ctx;
    d->stream = context_stream(ctx);
    d->device = context_device(ctx);
    d->fp64 = o->precision == AG_PREC_FP64;
    d->esz = d->fp64 ? sizeof(double) : sizeof(float);
    d->N = p->n_atoms;
    d->n_conf = n_conformers;
    d->n_maps = p->n_maps;
    d->floating = p->floating_grid ? 1 : 0;
    d->constriction = p->constriction_grid ? 1 : 0;
    d->cmap_cutoff = p->constriction_cutoff;
    d->n_out = d->n_maps + d->floating + d->constriction;
    d->n_atom_maps = nAM;
    d->elec = p->elec_map;
    d->need_h = need_h;
    d->P = (long long)p->n1[0] * p->n1[1] * p->n1[2];
    const int N = d->N, K = n_conformers;
    for (int k = 0; k < K; k++) {
        d->coord.insert(d->coord.end(), p->coord, p->coord + 3 * (size_t)N);
        d->charge.insert(d->charge.end(), p->charge, p->charge + N);
        d->rv.insert(d->rv.end(), p->rvector, p->rvector + 3 * (size_t)N);
        d->rv2.insert(d->rv2.end(), p->rvector2, p->rvector2 + 3 * (size_t)N);
    }
    std::vector<int> meta(std::max(N, 1), 0);
    for (int a = 0; a < N; a++) {
        const bool skip = p->disorder_h && p->disorder[a] && p->rec_type[a] == p->hydrogen_type;
        // without directional terms the hbond class changes nothing: drop it so
        // the kernels skip the angular factors
        const int hb = need_ang ? p->hbond[a] : 0;
        meta[a] = (p->rec_type[a] & DM_TYPE_MASK) | (hb << DM_HB_SHIFT) | ((p->rexp[a] & 7) << DM_REXP_SHIFT) |
                  (p->disorder[a] ? DM_DIS : 0) | (skip ? DM_SKIP : 0);
        if (p->hbond[a] == 1 || p->hbond[a] == 2) d->h_index.push_back(a);
    }

    DiffArgs &A = d->args;
    std::memset(&A, 0, sizeof A);
    A.need_ang = need_ang ? 1 : 0;
    A.n_atoms = N;
    A.n1x = p->n1[0]; A.n1y = p->n1[1]; A.n1z = p->n1[2];
    A.nex = p->ne[0]; A.ney = p->ne[1]; A.nez = p->ne[2];
    A.P = d->P;
    A.spacing = p->spacing;
    A.n_conf = K;
    A.disorder_h = p->disorder_h;
    A.hydrogen_type = p->hydrogen_type;
    A.n_rec_types = p->n_rec_types;
    A.n_atom_maps = nAM;
    A.solpar_q = p->solpar_q;
    A.n_h = (int)d->h_index.size();
    for (int i = 0; i < 3; i++) A.cov_pos[i] = p->cov_pos[i];
    A.cov_half_width = p->cov_half_width;
    A.cov_barrier = p->cov_barrier;
    A.elec_map = p->elec_map;
    A.n_slots = (int)slots.size();
    A.n_mm = n_mm;
    A.n_maps_out = d->n_out;  // per-conformer stride of the maps (energy maps, then fmap/cmap)
    A.tab_stride = std::max(4, (A.n_slots + 3) / 4 * 4);
    for (int s = 0; s < A.n_slots; s++) {
        const Slot &sl = slots[s];
        A.slot_map[s] = sl.map;
        A.slot_kind[s] = sl.kind;
        A.slot_tab[s] = sl.tab;
        A.slot_mm[s] = sl.mm ? s : -1;
        A.slot_desolv[s] = sl.desolv;
        A.slot_sp[s] = (sl.kind != DK_D) ? p->map_solpar_probe[sl.map] : 0.0;
        A.slot_vp[s] = (sl.kind != DK_D) ? p->map_vol_probe[sl.map] : 0.0;
        std::memcpy(A.act[s], sl.act, 16);
        if (sl.kind == DK_D || sl.desolv) A.need_sol = 1;
    }
    // cell list geometry: at most 6 cells per axis around a brick
    const double span = (DF_BRICK_X - 1) * p->spacing + 2 * DF_RADIUS;
    A.cell_size = std::max(4.0, span / 5.0);
    for (int i = 0; i < 3; i++) {
        const double lo = -p->ne[i] * p->spacing - DF_RADIUS, hi = (p->n1[i] - 1 - p->ne[i]) * p->spacing + DF_RADIUS;
        A.cell0[i] = lo;
        const int n = (int)std::ceil((hi - lo) / A.cell_size) + 1;
        if (i == 0) A.ncx = n; else if (i == 1) A.ncy = n; else A.ncz = n;
    }
    d->ncells = (size_t)A.ncx * A.ncy * A.ncz;
    const size_t NK = (size_t)N * K;

    DF_CK(d->alloc(&d->d_x, NK)); DF_CK(d->alloc(&d->d_y, NK)); DF_CK(d->alloc(&d->d_z, NK));
    DF_CK(d->alloc(&d->d_q, NK)); DF_CK(d->alloc(&d->d_vol, N)); DF_CK(d->alloc(&d->d_solpar, N));
    DF_CK(d->alloc(&d->d_rv, 3 * NK)); DF_CK(d->alloc(&d->d_rv2, 3 * NK));
    DF_CK(d->alloc(&d->d_meta, N)); DF_CK(d->alloc(&d->d_h, d->h_index.size()));
    DF_CK(d->alloc(&d->d_cell_start, (d->ncells + 1) * K)); DF_CK(d->alloc(&d->d_cell_atoms, NK));
    DF_CK(d->alloc(&d->d_ch, (size_t)d->P * K));
    DF_CK(d->alloc(&d->d_mmarg, 2 * (size_t)n_mm * d->P * K));
    DF_CK(d->alloc(&d->d_grad, 10 * NK));
    unsigned char *mp = nullptr;
    DF_CK(d->alloc(&mp, d->map_bytes())); d->d_maps = mp;
    DF_CK(cudaMemcpy(d->d_vol, p->vol, N * sizeof(double), cudaMemcpyHostToDevice));
    DF_CK(cudaMemcpy(d->d_solpar, p->solpar, N * sizeof(double), cudaMemcpyHostToDevice));
    DF_CK(cudaMemcpy(d->d_meta, meta.data(), N * sizeof(int), cudaMemcpyHostToDevice));
    if (!d->h_index.empty())
        DF_CK(cudaMemcpy(d->d_h, d->h_index.data(), d->h_index.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (d->fp64) {
        std::vector<R2<double>> vdw, sol, eps;
        build_tables(p, A, vdw, sol, eps);
        DF_CK(put(&d->d_vdw, vdw, d.get())); DF_CK(put(&d->d_sol, sol, d.get())); DF_CK(put(&d->d_eps, eps, d.get()));
    } else {
        std::vector<R2<float>> vdw, sol, eps;
        build_tables(p, A, vdw, sol, eps);
        DF_CK(put(&d->d_vdw, vdw, d.get())); DF_CK(put(&d->d_sol, sol, d.get())); DF_CK(put(&d->d_eps, eps, d.get()));
    }
    A.x = d->d_x; A.y = d->d_y; A.z = d->d_z; A.q = d->d_q; A.vol = d->d_vol; A.solpar = d->d_solpar;
    A.rv = d->d_rv; A.rv2 = d->d_rv2; A.meta = d->d_meta; A.h_index = d->d_h;
    A.cell_start = d->d_cell_start; A.cell_atoms = d->d_cell_atoms;
    for (auto &e : d->ev) DF_CK(cudaEventCreate(&e));
    for (int k = 0; k < K; k++) {
        st = d->upload_conformer(k);
        if (st != AG_OK) return st;
    }
    *out = d.release();
    return AG_OK;
}

ag_status ag_diff_create(ag_context *ctx, const ag_problem *p, const ag_opts *o, ag_diff **out)
{
    return ag_diff_create_batch(ctx, p, o, 1, out);
}

ag_status ag_diff_set_conformer(ag_diff *d, int32_t k, const double *coord, const double *charge,
                                const double *rvector, const double *rvector2)
{
    if (!d) { set_last_error("ag_diff_set_conformer: null argument"); return AG_ERR_INVALID; }
    if (k < 0 || k >= d->n_conf) { set_last_error("ag_diff_set_conformer: conformer out of range"); return AG_ERR_INVALID; }
    const size_t N = d->N, o1 = (size_t)k * N, o3 = 3 * o1;
    for (size_t i = 0; coord && i < 3 * N; i++)
        if (!std::isfinite(coord[i])) { set_last_error("ag_diff_set_atoms: non-finite coordinate"); return AG_ERR_INVALID; }
    for (size_t i = 0; charge && i < N; i++)
        if (!std::isfinite(charge[i])) { set_last_error("ag_diff_set_atoms: non-finite charge"); return AG_ERR_INVALID; }
    DF_CK(cudaSetDevice(d->device));
    const ag_status rs = d->refresh_host();
    if (rs != AG_OK) return rs;
    if (coord) std::copy(coord, coord + 3 * N, d->coord.begin() + o3);
    if (charge) std::copy(charge, charge + N, d->charge.begin() + o1);
    if (rvector) std::copy(rvector, rvector + 3 * N, d->rv.begin() + o3);
    if (rvector2) std::copy(rvector2, rvector2 + 3 * N, d->rv2.begin() + o3);
    return d->upload_conformer(k);
}

ag_status ag_diff_set_atoms(ag_diff *d, const double *coord, const double *charge, const double *rvector,
                            const double *rvector2)
{
    return ag_diff_set_conformer(d, 0, coord, charge, rvector, rvector2);
}

ag_status ag_diff_forward(ag_diff *d, int32_t keep_closest_h, void *device_out)
{
    if (!d) { set_last_error("ag_diff_forward: null argument"); return AG_ERR_INVALID; }
    if (device_out && !device_accessible(device_out, d->device)) {
        set_last_error("ag_diff_forward: device_out must be device memory of the object's GPU");
        return AG_ERR_INVALID;
    }
    DF_CK(cudaSetDevice(d->device));
    cudaStream_t s = d->stream;
    unsigned char *out = device_out ? (unsigned char *)device_out : (unsigned char *)d->d_maps;
    const DiffArgs &A = d->args;
    const bool search = !keep_closest_h || !d->have_ch;
    bool timed_search = false;
    if (search) {
        d->have_ch = false;
        if (d->need_h) {
            if (A.n_h == 0) {
                set_last_error("no closestH atom was found");  // main.cpp:3011-3014
                return AG_ERR_NO_CLOSEST_H;
            }
            DF_CK(cudaEventRecord(d->ev[4], s));
            DF_CK(launch_closest_h(A, d->d_ch, s));
            DF_CK(cudaEventRecord(d->ev[5], s));
            timed_search = true;
        } else {  // no map reads Hramp
            DF_CK(cudaMemsetAsync(d->d_ch, 0xff, sizeof(int) * (size_t)d->P * d->n_conf, s));
        }
    }
    DF_CK(cudaEventRecord(d->ev[0], s));
    if (d->elec >= 0) DF_CK(launch_emap_lin(d->fp64, A, d->d_eps, out + d->esz * d->P * d->elec, s));
    DF_CK(launch_near_lin(d->fp64, A, d->d_vdw, d->d_sol, out, d->d_ch, d->d_mmarg, s));
    if (d->floating || d->constriction)
        for (int k = 0; k < d->n_conf; k++) {
            // floating and constriction grids of conformer k (FP64, the reference's distances)
            unsigned char *base = out + d->esz * (size_t)d->P * ((size_t)k * d->n_out + d->n_maps);
            unsigned char *fm = d->floating ? base : nullptr;
            unsigned char *cm = d->constriction ? base + d->esz * (size_t)d->P * d->floating : nullptr;
            if (d->fp64)
                DF_CK(launch_distance_maps(d->conformer_geometry(k), d->cmap_cutoff, nullptr, nullptr, (double *)fm,
                                           (double *)cm, s));
            else
                DF_CK(launch_distance_maps(d->conformer_geometry(k), d->cmap_cutoff, (float *)fm, (float *)cm, nullptr,
                                           nullptr, s));
        }
    DF_CK(cudaEventRecord(d->ev[1], s));
    DF_CK(cudaStreamSynchronize(s));
    DF_CK(cudaEventElapsedTime(&d->fwd_ms, d->ev[0], d->ev[1]));
    d->ch_ms = 0;
    if (timed_search) DF_CK(cudaEventElapsedTime(&d->ch_ms, d->ev[4], d->ev[5]));
    d->have_ch = true;
    d->have_fwd = true;
    return AG_OK;
}

const void *ag_diff_device_maps(const ag_diff *d) { return d ? d->d_maps : nullptr; }

ag_status ag_diff_download(ag_diff *d, void *host_maps)
{
    if (!d || !host_maps) { set_last_error("ag_diff_download: null argument"); return AG_ERR_INVALID; }
    DF_CK(cudaSetDevice(d->device));
    DF_CK(cudaMemcpyAsync(host_maps, d->d_maps, d->map_bytes(), cudaMemcpyDeviceToHost, d->stream));
    DF_CK(cudaStreamSynchronize(d->stream));
    return AG_OK;
}

ag_status ag_diff_closest_h(ag_diff *d, int32_t *host_out)
{
    if (!d || !host_out) { set_last_error("ag_diff_closest_h: null argument"); return AG_ERR_INVALID; }
    if (!d->have_ch) { set_last_error("ag_diff_closest_h: no forward yet"); return AG_ERR_INVALID; }
    DF_CK(cudaSetDevice(d->device));
    DF_CK(cudaMemcpyAsync(host_out, d->d_ch, sizeof(int) * (size_t)d->P * d->n_conf, cudaMemcpyDeviceToHost,
                          d->stream));
    DF_CK(cudaStreamSynchronize(d->stream));
    return AG_OK;
}

ag_status ag_diff_backward(ag_diff *d, const void *grad_maps, int32_t grad_on_device, double *g_coord,
                           double *g_charge, double *g_rvector, double *g_rvector2)
{
    if (!d || !grad_maps) { set_last_error("ag_diff_backward: null argument"); return AG_ERR_INVALID; }
    if (!d->have_fwd) { set_last_error("ag_diff_backward: no forward to differentiate"); return AG_ERR_INVALID; }
    if (grad_on_device && !device_accessible(grad_maps, d->device)) {
        set_last_error("ag_diff_backward: grad_maps is not device memory of the object's GPU");
        return AG_ERR_INVALID;
    }
    DF_CK(cudaSetDevice(d->device));
    cudaStream_t s = d->stream;
    const size_t N = d->N, K = d->n_conf;
    const unsigned char *gm = (const unsigned char *)grad_maps;
    if (!grad_on_device) {
        if (!d->d_gmaps) {
            unsigned char *gp = nullptr;
            DF_CK(d->alloc(&gp, d->map_bytes()));
            d->d_gmaps = gp;
        }
        DF_CK(cudaMemcpyAsync(d->d_gmaps, grad_maps, d->map_bytes(), cudaMemcpyHostToDevice, s));
        gm = (const unsigned char *)d->d_gmaps;
    }
    DiffGrads g;
    g.xyz = d->d_grad;
    g.q = d->d_grad + 3 * N;
    g.rv = d->d_grad + 4 * N;
    g.rv2 = d->d_grad + 7 * N;
    DF_CK(cudaMemsetAsync(d->d_grad, 0, 10 * N * K * sizeof(double), s));
    DF_CK(cudaEventRecord(d->ev[2], s));
    if (d->elec >= 0) DF_CK(launch_emap_lin_adj(d->fp64, d->args, d->d_eps, gm + d->esz * d->P * d->elec, g, s));
    DF_CK(launch_near_lin_adj(d->fp64, d->args, d->d_vdw, d->d_sol, gm, d->d_ch, d->d_mmarg, g, s));
    if (d->floating)  // the constriction grid is piecewise constant: no gradient
        for (size_t k = 0; k < K; k++)
            DF_CK(launch_fmap_adjoint(d->conformer_geometry((int)k),
                                      gm + d->esz * (size_t)d->P * (k * d->n_out + d->n_maps), d->fp64,
                                      d->d_grad + 10 * N * k, s));
    DF_CK(cudaEventRecord(d->ev[3], s));
    for (size_t k = 0; k < K; k++) {
        const double *base = d->d_grad + 10 * N * k;
        if (g_coord) DF_CK(cudaMemcpyAsync(g_coord + 3 * N * k, base, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (g_charge) DF_CK(cudaMemcpyAsync(g_charge + N * k, base + 3 * N, N * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (g_rvector)
            DF_CK(cudaMemcpyAsync(g_rvector + 3 * N * k, base + 4 * N, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (g_rvector2)
            DF_CK(cudaMemcpyAsync(g_rvector2 + 3 * N * k, base + 7 * N, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    DF_CK(cudaStreamSynchronize(s));
    DF_CK(cudaEventElapsedTime(&d->bwd_ms, d->ev[2], d->ev[3]));
    return AG_OK;
}

ag_status ag_diff_set_bonds(ag_diff *d, const int32_t *topo)
{
    if (!d || !topo) { set_last_error("ag_diff_set_bonds: null argument"); return AG_ERR_INVALID; }
    const int N = d->N;
    for (int a = 0; a < N; a++) {
        const int32_t *t = topo + 7 * (size_t)a;
        const int kind = t[0];
        bool ok = kind >= AG_BOND_NONE && kind <= AG_BOND_A1;
        auto in = [&](int32_t i) { return i >= 0 && i < N; };
        if (ok && (kind == AG_BOND_D1 || kind == AG_BOND_A2_ONE || kind == AG_BOND_A2_DIS || kind == AG_BOND_A2_TWO))
            ok = in(t[1]);
        if (ok && kind == AG_BOND_A2_TWO) ok = in(t[2]);
        if (ok && kind == AG_BOND_A2_ONE) ok = t[2] == -1 || in(t[2]);
        if (ok && kind == AG_BOND_A1) {
            ok = t[3] >= 0 && t[3] <= 3;
            for (int b = 0; ok && b < t[3]; b++) ok = in(t[4 + b]);
        }
        if (!ok) { set_last_error("ag_diff_set_bonds: invalid topology entry"); return AG_ERR_INVALID; }
    }
    DF_CK(cudaSetDevice(d->device));
    if (!d->d_topo) DF_CK(d->alloc(&d->d_topo, 7 * (size_t)std::max(N, 1)));
    DF_CK(cudaMemcpyAsync(d->d_topo, topo, 7 * (size_t)N * sizeof(int32_t), cudaMemcpyHostToDevice, d->stream));
    DF_CK(cudaStreamSynchronize(d->stream));
    return AG_OK;
}

ag_status ag_diff_set_atoms_device(ag_diff *d, const double *coord, const double *charge)
{
    if (!d || !coord) { set_last_error("ag_diff_set_atoms_device: null argument"); return AG_ERR_INVALID; }
    if (!device_accessible(coord, d->device) || (charge && !device_accessible(charge, d->device))) {
        set_last_error("ag_diff_set_atoms_device: coord and charge must be device memory of the object's GPU");
        return AG_ERR_INVALID;
    }
    DF_CK(cudaSetDevice(d->device));
    cudaStream_t s = d->stream;
    const int N = d->N, K = d->n_conf;
    const size_t NK = (size_t)N * K;
    if (!d->d_bad) {
        DF_CK(d->alloc(&d->d_bad, 1));
        DF_CK(d->alloc(&d->d_cell_of, std::max<size_t>(NK, 1)));
        DF_CK(d->alloc(&d->d_cell_count, std::max<size_t>(d->ncells * K, 1)));
    }
    DF_CK(cudaMemsetAsync(d->d_bad, 0, sizeof(int), s));
    DF_CK(launch_split_atoms((long long)NK, coord, charge, d->d_x, d->d_y, d->d_z, d->d_q, d->d_bad, s));
    int bad = 0;
    DF_CK(cudaMemcpyAsync(&bad, d->d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    DF_CK(cudaStreamSynchronize(s));
    d->host_stale = true;  // the split already replaced the device coordinates
    if (bad) {
        set_last_error("ag_diff_set_atoms_device: non-finite coordinate or charge");
        return AG_ERR_INVALID;
    }
    if (d->d_topo) DF_CK(launch_bond_vectors(K, N, d->d_topo, d->d_x, d->d_y, d->d_z, d->d_rv, d->d_rv2, s));
    DF_CK(launch_cell_lists(d->args, d->d_cell_of, d->d_cell_count, s));
    DF_CK(cudaStreamSynchronize(s));
    return AG_OK;
}

ag_status ag_diff_backward_device(ag_diff *d, const void *grad_maps, double *g_coord, double *g_charge)
{
    if (!d || !grad_maps) { set_last_error("ag_diff_backward_device: null argument"); return AG_ERR_INVALID; }
    if ((g_coord && !device_accessible(g_coord, d->device)) || (g_charge && !device_accessible(g_charge, d->device))) {
        set_last_error("ag_diff_backward_device: g_coord and g_charge must be device memory of the object's GPU");
        return AG_ERR_INVALID;
    }
    ag_status st = ag_diff_backward(d, grad_maps, 1, nullptr, nullptr, nullptr, nullptr);
    if (st != AG_OK) return st;
    cudaStream_t s = d->stream;
    const size_t N = d->N, K = d->n_conf;
    for (size_t k = 0; k < K; k++) {
        const double *base = d->d_grad + 10 * N * k;
        if (g_coord)
            DF_CK(cudaMemcpyAsync(g_coord + 3 * N * k, base, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, s));
        if (g_charge)
            DF_CK(cudaMemcpyAsync(g_charge + N * k, base + 3 * N, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    if (g_coord && d->d_topo)
        DF_CK(launch_bond_vectors_adj((int)K, (int)N, d->d_topo, d->d_x, d->d_y, d->d_z, d->d_grad, g_coord, s));
    DF_CK(cudaStreamSynchronize(s));
    return AG_OK;
}

ag_status ag_diff_timing(const ag_diff *d, float *forward_ms, float *closest_h_ms, float *backward_ms)
{
    if (!d) { set_last_error("ag_diff_timing: null argument"); return AG_ERR_INVALID; }
    if (forward_ms) *forward_ms = d->fwd_ms;
    if (closest_h_ms) *closest_h_ms = d->ch_ms;
    if (backward_ms) *backward_ms = d->bwd_ms;
    return AG_OK;
}

int32_t ag_diff_conformers(const ag_diff *d) { return d ? d->n_conf : 0; }

ag_status ag_diff_destroy(ag_diff *d)
{
    delete d;
    return AG_OK;
}

}  // extern "C"
