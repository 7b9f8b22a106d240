// C ABI of the hot path: contexts, plans and the kernel sequence that
// replaces the reference's grid-point loop (main.cpp:2805-3464).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "autogrid_b200.h"
#include "autogrid_b200_diag.h"
#include "kernels/kernels.h"
#include "kernels/maptext.h"
#include "kernels/tables.h"

namespace agb {
void set_last_error(const std::string &m);
}

using namespace agb;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

// Device blocks that finished arenas give back to their context, so that
// repeated batches reuse memory instead of calling cudaMalloc/cudaFree (which
// maps and unmaps pages, and synchronises) every time.  Freed with the
// context.  Thread-safe.
struct BlockCache {
    std::vector<std::pair<void *, size_t>> free;
    std::mutex mu;
    ~BlockCache()
    {
        for (auto &b : free) cudaFree(b.first);
    }
    cudaError_t take(size_t bytes, void **out, size_t *got)
    {
        {
            std::lock_guard<std::mutex> lock(mu);
            size_t best = free.size();
            for (size_t i = 0; i < free.size(); i++)
                if (free[i].second >= bytes && (best == free.size() || free[i].second < free[best].second)) best = i;
            if (best < free.size()) {
                *out = free[best].first;
                *got = free[best].second;
                free.erase(free.begin() + (long)best);
                return cudaSuccess;
            }
        }
        *got = bytes;
        return cudaMalloc(out, bytes);
    }
    void give(void *p, size_t bytes)
    {
        std::lock_guard<std::mutex> lock(mu);
        free.emplace_back(p, bytes);
    }
    size_t bytes()
    {
        std::lock_guard<std::mutex> lock(mu);
        size_t n = 0;
        for (auto &b : free) n += b.second;
        return n;
    }
    // Frees every cached block; returns the bytes freed.
    size_t release()
    {
        std::lock_guard<std::mutex> lock(mu);
        size_t n = 0;
        for (auto &b : free) {
            cudaFree(b.first);
            n += b.second;
        }
        free.clear();
        return n;
    }
};

// Bump allocator over a few large device blocks, released together: the
// buffers of a batch's instance plans (one block per 256 MiB instead of one
// cudaMalloc per buffer per instance).  Blocks come from and go back to the
// context's cache when it has one.  Thread-safe.
struct Arena {
    std::vector<std::pair<void *, size_t>> blocks;
    BlockCache *cache = nullptr;
    char *cur = nullptr;
    size_t left = 0;
    std::mutex mu;
    static constexpr size_t kBlock = size_t(256) << 20, kAlign = 256;
    explicit Arena(BlockCache *c = nullptr) : cache(c) {}
    ~Arena()
    {
        for (auto &b : blocks) {
            if (cache) cache->give(b.first, b.second);
            else cudaFree(b.first);
        }
    }
    cudaError_t alloc(size_t bytes, void **out)
    {
        bytes = (bytes + kAlign - 1) / kAlign * kAlign;
        std::lock_guard<std::mutex> lock(mu);
        if (bytes > left) {
            void *b = nullptr;
            size_t sz = std::max(bytes, kBlock);
            cudaError_t e = cache ? cache->take(sz, &b, &sz) : cudaMalloc(&b, sz);
            if (e != cudaSuccess) return e;
            blocks.emplace_back(b, sz);
            cur = (char *)b;
            left = sz;
        }
        *out = cur;
        cur += bytes;
        left -= bytes;
        return cudaSuccess;
    }
};

// Grow-only device buffers keyed by role; a context keeps one set so repeated
// one-shot calls do not re-allocate.  With an arena, buffers come from it and
// are released with it.
struct BufferSet {
    std::map<std::string, DevBuf> bufs;
    Arena *arena = nullptr;
    ~BufferSet()
    {
        if (arena) return;
        for (auto &kv : bufs)
            if (kv.second.p) cudaFree(kv.second.p);
    }
    cudaError_t ensure(const std::string &name, size_t bytes, void **out)
    {
        DevBuf &b = bufs[name];
        if (bytes == 0) bytes = 16;
        if (b.cap < bytes) {
            if (b.p && !arena) cudaFree(b.p);
            b.p = nullptr;
            b.cap = 0;
            cudaError_t e = arena ? arena->alloc(bytes, &b.p) : cudaMalloc(&b.p, bytes);
            if (e != cudaSuccess) return e;
            b.cap = bytes;
        }
        *out = b.p;
        return cudaSuccess;
    }
};

// Makes a device current for the scope of an entry point and gives the
// caller's current device back on return.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int device)
    {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

ag_status cuda_fail(cudaError_t e, const char *what)
{
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return AG_ERR_CUDA;
}

#define AGB_CK(call)                                   \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

ag_status invalid(const std::string &m)
{
    set_last_error(m);
    return AG_ERR_INVALID;
}

// Device statistics counters of a context (and of a batch):
//   context: [0] near pairs, [1] FP64 fallbacks, [2..4] far-field bin guard
//            (FarArgs::edge_counters);
//   batch:   [0] far work units, [1] near work units, [2..3] near statistics,
//            [4..6] far-field bin guard.
constexpr int kCounters = 8;

// One-shot calls: z-slab height of the copy/compute pipeline (whole far-field
// frames and near-field brick rows) and the most slabs one call uses.
// 24 planes: 13.74 ms end to end for 127^3 points x 16 maps, against 13.85 ms
// with 16 and 14.08 ms with 32.
constexpr int kSlabZ = 24;
constexpr int kMaxSlabs = 16;

int slab_count(const DevProblem &d) { return std::min(kMaxSlabs, (d.n1z + kSlabZ - 1) / kSlabZ); }
// z planes [z0, z1) of slab k: kSlabZ planes each, the last one to n1z
void slab_range(const DevProblem &d, int k, int *z0, int *z1)
{
    *z0 = kSlabZ * k;
    *z1 = k == slab_count(d) - 1 ? d.n1z : *z0 + kSlabZ;
}

}  // namespace

struct ag_context {
    int device = 0;
    int sms = 148;  // streaming multiprocessors of the device (queried at creation)
    cudaStream_t stream = nullptr;
    // the far-field kernel runs on `side`, concurrently with the near-field
    // kernel, forked from and joined back to the caller's stream by events
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // one-shot calls copy finished z-slabs of the maps back on `copy` while
    // later slabs compute (per-slab completion events)
    cudaStream_t copy = nullptr;
    std::vector<cudaEvent_t> far_done, red_done;
    cudaEvent_t copy_done = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evf0 = nullptr, evf1 = nullptr;
    // evfx: between the far-field kernel and its fix-up; evn0/evn1: around
    // the near-field launches (run_plan only)
    cudaEvent_t evfx = nullptr, evn0 = nullptr, evn1 = nullptr;
    bool had_near = false, had_fixup_event = false;
    ag_stats stats{};
    BufferSet pool;
    unsigned long long *d_counters = nullptr;
    // device blocks of finished batch arenas, reused by later batches
    BlockCache blocks;
    // map text (ag_maps_format): device scratch and text, pinned host copy
    BufferSet text_bufs;
    char *h_text = nullptr;
    size_t h_text_cap = 0;
    cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};  // measure and write passes
    BufferSet table_bufs;  // ag_tables_build
    // the last run, whose statistics ag_context_stats() settles
    bool pending = false, had_far = false;
    int last_launches = 0;
    int64_t last_far_pairs = 0;
};

struct ag_plan {
    ag_context *ctx = nullptr;
    std::unique_ptr<BufferSet> own;
    BufferSet *bufs = nullptr;
    ag_opts opts{};
    DevProblem dp{};
    std::vector<NearGroup> groups;
    int mpad = 4, n_chunks = 0, chunk_atoms = 0;
    bool any_cov = false;
    int floating = 0, constriction = 0;  // distance maps after the n_maps energy maps
    int far_mode = FAR_TAB_TABLE;        // how k_emap_far obtains far table values (FarArgs::tab_mode)
    int tab_len = AG_NDIEL, far_clamp = 1;  // shared-memory far table (FarArgs::tab_len, clamp)
    float far_const = 0.f;
    double constriction_cutoff = 7.5;
    float *maps32 = nullptr;
    double *maps64 = nullptr;
    double *cov = nullptr;
    float *far_partial = nullptr;
    uint32_t *edge_bits = nullptr;     // far-field bin guard: per (thread, atom) edge bits (FarArgs::edge_bits)
    ReduceInst *d_reduce = nullptr;    // e-map reduction of this plan (one instance)
    long long *d_reduce_begin = nullptr;
    double *x128 = nullptr, *y128 = nullptr, *z128 = nullptr;
    float *qw = nullptr, *far_tab = nullptr, *etab = nullptr, *solf = nullptr, *vdwT = nullptr;
    float4 *atomA = nullptr, *atomB = nullptr;
    int *meta = nullptr;
    size_t h2d_bytes = 0;
    int last_launches = 0;
    int far_early = 0;  // far-field slabs a one-shot call launched while its plan was still being built
};

namespace {

// Validate an ag_problem against the limits of the reference build.  The
// reference's grids are symmetric: n1 odd and ne = (n1-1)/2 (check_size.cpp:
// 79-83, main.cpp:1083-1097).  symmetric = false accepts any box (n1 >= 1,
// any offset ne), such as a z-slab of a grid (the differentiable mode's shards).
ag_status validate(const ag_problem *p, bool symmetric = true)
{
    if (!p) return invalid("null problem");
    if (p->n_atoms < 0 || p->n_atoms > AG_MAX_ATOMS) {
        set_last_error("n_atoms out of range [0, AG_MAX_ATOMS]");
        return AG_ERR_TOO_LARGE;
    }
    for (int i = 0; i < 3; i++) {
        if (!symmetric) {
            if (p->n1[i] < 1 || p->n1[i] > AG_MAX_GRID_PTS + 1 || p->ne[i] < -(1 << 20) || p->ne[i] > (1 << 20))
                return invalid("n1 must be within [1, MAX_GRID_PTS+1] and |ne| <= 2^20");
            continue;
        }
        if (p->n1[i] < 1 || p->n1[i] > AG_MAX_GRID_PTS + 1 || (p->n1[i] % 2) != 1)
            return invalid("n1 must be odd and within [1, MAX_GRID_PTS+1]");
        if (p->ne[i] != (p->n1[i] - 1) / 2) return invalid("ne must equal (n1-1)/2");
    }
    if (!(p->spacing > 0.0) || !std::isfinite(p->spacing)) return invalid("spacing must be positive");
    if (p->n_maps < 1 || p->n_maps > AG_MAX_MAPS) return invalid("n_maps out of range [1, MAX_MAPS]");
    if (p->n_atom_maps < 0 || p->n_atom_maps > p->n_maps) return invalid("n_atom_maps out of range");
    if (p->elec_map >= p->n_maps || (p->elec_map >= 0 && p->elec_map < p->n_atom_maps))
        return invalid("elec_map index out of range");
    if (p->dsolv_map >= p->n_maps || (p->dsolv_map >= 0 && p->dsolv_map < p->n_atom_maps))
        return invalid("dsolv_map index out of range");
    if (p->elec_map >= 0 && p->elec_map == p->dsolv_map) return invalid("elec_map == dsolv_map");
    if (p->n_atom_maps + (p->elec_map >= 0) + (p->dsolv_map >= 0) != p->n_maps)
        return invalid("n_maps != n_atom_maps + elec + dsolv");
    if (p->n_rec_types < 0 || p->n_rec_types > AG_MAX_REC_TYPES) return invalid("n_rec_types out of range");
    if (p->constriction_grid && !std::isfinite(p->constriction_cutoff)) return invalid("constriction_cutoff must be finite");
    const int N = p->n_atoms;
    if (N > 0 && (!p->coord || !p->charge || !p->vol || !p->solpar || !p->rec_type || !p->hbond || !p->rexp ||
                  !p->rvector || !p->rvector2 || !p->disorder))
        return invalid("null atom array");
    if (p->n_atom_maps > 0 && (!p->map_is_covalent || !p->map_is_hbonder || !p->map_hbond ||
                               !p->map_solpar_probe || !p->map_vol_probe || !p->e_vdw_hb))
        return invalid("null map array");
    if (!p->sol_fn || (p->dddiel && !p->r_epsilon_fn)) return invalid("null table");
    int n_h = 0;
    for (int a = 0; a < N; a++) {
        if (p->rec_type[a] < 0 || p->rec_type[a] >= std::max(p->n_rec_types, 1)) return invalid("rec_type out of range");
        if (p->hbond[a] < 0 || p->hbond[a] > 6) return invalid("hbond class out of range");
        for (int k = 0; k < 3; k++)
            if (!std::isfinite(p->coord[3 * a + k])) return invalid("non-finite coordinate");
        if (!std::isfinite(p->charge[a])) return invalid("non-finite charge");
        if (p->hbond[a] == 1 || p->hbond[a] == 2) n_h++;
    }
    if (p->disorder_h && p->hydrogen_type >= std::max(p->n_rec_types, 1)) return invalid("hydrogen_type out of range");
    if (p->n_atom_maps > 0 && n_h == 0) {
        set_last_error("no closestH atom was found");  // main.cpp:3011-3014
        return AG_ERR_NO_CLOSEST_H;
    }
    return AG_OK;
}

}  // namespace

// Internal accessors for the other host modules of the library.
namespace agb {
ag_status validate_problem(const ag_problem *p) { return validate(p); }
ag_status validate_problem_box(const ag_problem *p) { return validate(p, false); }
cudaStream_t context_stream(const ag_context *c) { return c->stream; }
int context_device(const ag_context *c) { return c->device; }
// True when kernels on `device` may dereference ptr: device memory of that
// GPU or managed memory.  Entry points that hand a caller's pointer to a
// kernel check it first, so a host pointer is an argument error, not a fault.
bool device_accessible(const void *ptr, int device)
{
    if (!ptr) return false;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == device);
}
}  // namespace agb

namespace {

// True for memory that only the device can read (cudaMalloc'd); host,
// pinned and managed memory are read on the host.
bool is_device_memory(const void *ptr)
{
    if (!ptr) return false;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice;
}

template <class T>
cudaError_t upload(BufferSet *b, const char *name, const T *src, size_t n, T **dst, cudaStream_t s, size_t *acc)
{
    void *d = nullptr;
    cudaError_t e = b->ensure(name, n * sizeof(T), &d);
    if (e != cudaSuccess) return e;
    *dst = (T *)d;
    if (n) {
        e = cudaMemcpyAsync(d, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
        if (acc) *acc += n * sizeof(T);
    }
    return e;
}

// Build the device image of a problem (host work is O(atoms + tables)).
ag_status launch_far_slab(ag_plan *pl, cudaStream_t s, int k, int nslab);

// pipelined: far-field chunking sized per kSlabZ-plane slab (one-shot calls and
// z-slab runs); early_far: with pipelined, also launch far slab 0 from here.
ag_status build_plan(ag_plan *pl, const ag_problem *p, cudaStream_t s, bool pipelined, bool early_far = true)
{
    ag_status st = validate(p);
    if (st != AG_OK) return st;
    BufferSet *B = pl->bufs;
    DevProblem &d = pl->dp;
    std::memset(&d, 0, sizeof d);
    const int N = p->n_atoms, nAM = p->n_atom_maps;
    d.n_atoms = N; d.n_maps = p->n_maps; d.n_atom_maps = nAM; d.n_rec_types = p->n_rec_types;
    d.elec_map = p->elec_map; d.dsolv_map = p->dsolv_map;
    d.n1x = p->n1[0]; d.n1y = p->n1[1]; d.n1z = p->n1[2];
    d.nex = p->ne[0]; d.ney = p->ne[1]; d.nez = p->ne[2];
    d.P = (long long)d.n1x * d.n1y * d.n1z;
    d.spacing = p->spacing;
    d.dddiel = p->dddiel; d.disorder_h = p->disorder_h; d.hydrogen_type = p->hydrogen_type;
    d.sep_desolv = p->separate_desolvation_maps;
    d.invdielcal = p->invdielcal; d.coeff_estat = p->coeff_estat; d.solpar_q = p->solpar_q;
    for (int i = 0; i < 3; i++) d.cov_pos[i] = p->cov_pos[i];
    d.cov_half_width = p->cov_half_width; d.cov_barrier = p->cov_barrier;
    d.report_collisions = p->report_collisions ? 1 : 0;
    pl->h2d_bytes = 0;
    size_t *acc = &pl->h2d_bytes;

    const bool dev_tables = is_device_memory(p->e_vdw_hb);
    if (dev_tables != is_device_memory(p->sol_fn) || (p->dddiel && dev_tables != is_device_memory(p->r_epsilon_fn)))
        return invalid("the problem's tables must all be host memory or all device memory");

    // far-field inputs first: atoms as x*A_DIV and weighted charges, the far
    // table, the chunking and the partial sums.  A slab-pipelined one-shot run
    // launches its first far-field slab from here, so that the GPU computes
    // while the rest of the plan is built on the host.
    std::vector<double> x(N), y(N), z(N), x128(N), y128(N), z128(N);
    std::vector<float> qw(N);
    for (int a = 0; a < N; a++) {
        x[a] = p->coord[3 * a]; y[a] = p->coord[3 * a + 1]; z[a] = p->coord[3 * a + 2];
        x128[a] = x[a] * AG_A_DIV; y128[a] = y[a] * AG_A_DIV; z128[a] = z[a] * AG_A_DIV;
        qw[a] = (float)(p->charge[a] * p->coeff_estat * AG_A_DIV);
    }
    // The far kernel's table length: past the largest distance (bins) from an
    // atom to any point the kernel evaluates -- the box padded to whole
    // frames, whose points past the box are computed and not stored -- so
    // that no pair's bin needs a clamp; the bins from NDIEL-1 on repeat its
    // value (the reference clamps the bin, main.cpp:2956).  Beyond FAR_TAB_MAX
    // the kernel clamps t instead.
    {
        const int padded[3] = {frames_x(p->n1[0]) * FRAME_X, frames_y(p->n1[1]) * FRAME_Y, frames_z(p->n1[2]) * FRAME_Z};
        double dmax2 = 0.0;
        for (int a = 0; a < N; a++) {
            double d2 = 0.0;
            for (int i = 0; i < 3; i++) {
                const double c = i == 0 ? x[a] : (i == 1 ? y[a] : z[a]);
                const double lo_c = (double)(-p->ne[i]) * p->spacing;
                const double hi_c = (double)(padded[i] - 1 - p->ne[i]) * p->spacing;
                const double dd = std::max(std::fabs(c - lo_c), std::fabs(c - hi_c));
                d2 += dd * dd;
            }
            dmax2 = std::max(dmax2, d2);
        }
        const double tmax = std::sqrt(dmax2) * AG_A_DIV * (1.0 + 1.0e-5) + 8.0;
        if (tmax < (double)FAR_TAB_MAX - 4.0) {
            pl->far_clamp = 0;
            pl->tab_len = ((int)std::ceil(tmax) + 4) / 4 * 4;
        } else {
            pl->far_clamp = 1;
            pl->tab_len = AG_NDIEL;
        }
    }
    const int TL = pl->tab_len;
    std::vector<float> far_tab;
    if (!dev_tables) {
        // [0, tab_len): the far kernel's table, zero below FAR_BIN0 (those
        // pairs are the near kernel's), bin NDIEL-1 repeated past it;
        // [tab_len, tab_len + NDIEL): the whole table, for far pairs whose
        // exact bin the bin guard finds below FAR_BIN0
        far_tab.assign((size_t)TL + AG_NDIEL, 0.f);
        for (int k = 0; k < AG_NDIEL; k++) far_tab[TL + k] = (float)(p->dddiel ? p->r_epsilon_fn[k] : p->invdielcal);
        for (int k = AG_NEINT; k < TL; k++) far_tab[k] = far_tab[TL + std::min(k, AG_NDIEL - 1)];
        // a constant dielectric needs no far-field table gather
        if (!p->dddiel) {
            pl->far_mode = FAR_TAB_CONST;
            pl->far_const = (float)p->invdielcal;
        }
    }
    // far-field chunking: enough CTAs for ~8 waves per launch; a slab-pipelined
    // one-shot run launches one slab of frames at a time, ~3 waves each
    const long long frames = pipelined ? (long long)frames_x(d.n1x) * frames_y(d.n1y) * (kSlabZ / FRAME_Z)
                                       : (long long)frames_x(d.n1x) * frames_y(d.n1y) * frames_z(d.n1z);
    const int tile = 512;
    if (p->elec_map >= 0 && N > 0) {
        const long long sms = pl->ctx ? pl->ctx->sms : 148;
        const long long target = pipelined ? sms * 3 * 3 : sms * 3 * 8;
        int nch = (int)std::max(1LL, (target + frames - 1) / frames);
        nch = std::min(nch, (N + tile - 1) / tile);
        pl->chunk_atoms = ((N + nch - 1) / nch + tile - 1) / tile * tile;
        pl->n_chunks = (N + pl->chunk_atoms - 1) / pl->chunk_atoms;
    } else {
        pl->chunk_atoms = 0;
        pl->n_chunks = 0;
    }
    void *v = nullptr;
    const size_t P = (size_t)d.P;
    if (pl->n_chunks > 0 && pl->opts.precision != AG_PREC_FP64) {
        AGB_CK(B->ensure("far_partial", (size_t)pl->n_chunks * P * sizeof(float), &v));
        pl->far_partial = (float *)v;
    } else {
        pl->far_partial = nullptr;
    }
    pl->edge_bits = nullptr;
    if (pl->far_partial && pl->far_mode != FAR_TAB_CONST) {
        const int nframes = frames_x(d.n1x) * frames_y(d.n1y) * frames_z(d.n1z);
        AGB_CK(B->ensure("edge_bits", far_edge_bits_bytes(pl->n_chunks, pl->chunk_atoms, nframes), &v));
        pl->edge_bits = (uint32_t *)v;
    }
    AGB_CK(upload(B, "x128", x128.data(), N, &pl->x128, s, acc));
    AGB_CK(upload(B, "y128", y128.data(), N, &pl->y128, s, acc));
    AGB_CK(upload(B, "z128", z128.data(), N, &pl->z128, s, acc));
    AGB_CK(upload(B, "qw", qw.data(), N, &pl->qw, s, acc));
    if (!dev_tables) AGB_CK(upload(B, "far_tab", far_tab.data(), far_tab.size(), &pl->far_tab, s, acc));
    pl->far_early = 0;
    if (pipelined && early_far && !dev_tables && pl->far_partial && d.elec_map >= 0) {
        // the run's statistics start here: counters cleared, then ev0, then the fork
        ag_context *c = pl->ctx;
        AGB_CK(cudaMemsetAsync(c->d_counters, 0, kCounters * sizeof(unsigned long long), s));
        AGB_CK(cudaEventRecord(c->ev0, s));
        ag_status st = launch_far_slab(pl, s, 0, slab_count(d));
        if (st != AG_OK) return st;
        pl->far_early = 1;
    }

    // the near kernel's staged atom record: bond vectors + vol, lone-pair
    // normal + desolvation factor, and packed metadata (type, hbond, rexp, flags)
    std::vector<float4> atomA(std::max(N, 1)), atomB(std::max(N, 1));
    std::vector<int> meta(std::max(N, 1), 0);
    for (int a = 0; a < N; a++) {
        const double *rv = p->rvector + 3 * a, *rv2 = p->rvector2 + 3 * a;
        atomA[a] = make_float4((float)rv[0], (float)rv[1], (float)rv[2], (float)p->vol[a]);
        atomB[a] = make_float4((float)rv2[0], (float)rv2[1], (float)rv2[2],
                               (float)(p->solpar[a] + p->solpar_q * std::fabs(p->charge[a])));
        int m = (p->rec_type[a] & 31) | ((p->hbond[a] & 7) << 5) | ((p->rexp[a] & 7) << 8);
        if (p->disorder[a]) m |= 1 << 11;
        if (rv[0] == 0.0 && rv[1] == 0.0 && rv[2] == 0.0) m |= 1 << 12;
        if (p->disorder_h && p->disorder[a] && p->rec_type[a] == p->hydrogen_type) m |= 1 << 13;
        meta[a] = m;
    }
    std::vector<int> h_index;
    for (int a = 0; a < N; a++)
        if (p->hbond[a] == 1 || p->hbond[a] == 2) h_index.push_back(a);

    // cell list over the grid box grown by the near radius
    const double rc = AGB_NEAR_RADIUS, cs = AGB_CELL;
    double lo[3], hi[3];
    int nc[3];
    for (int i = 0; i < 3; i++) {
        lo[i] = (double)(-p->ne[i]) * p->spacing - rc;
        hi[i] = (double)(p->n1[i] - 1 - p->ne[i]) * p->spacing + rc;
        nc[i] = std::max(1, (int)std::ceil((hi[i] - lo[i]) / cs));
        d.cell0[i] = lo[i];
    }
    d.ncx = nc[0]; d.ncy = nc[1]; d.ncz = nc[2];
    d.cell_size = cs;
    const size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
    std::vector<int> cell_of(N, -1), cell_start(ncell + 1, 0), cell_atoms;
    for (int a = 0; a < N; a++) {
        const double c3[3] = {x[a], y[a], z[a]};
        int ci[3];
        bool in = true;
        for (int i = 0; i < 3; i++) {
            if (!(c3[i] >= lo[i] && c3[i] <= hi[i])) { in = false; break; }
            ci[i] = std::min(nc[i] - 1, (int)std::floor((c3[i] - lo[i]) / cs));
        }
        if (!in) continue;
        cell_of[a] = (ci[2] * nc[1] + ci[1]) * nc[0] + ci[0];
        cell_start[cell_of[a] + 1]++;
    }
    for (size_t c = 0; c < ncell; c++) cell_start[c + 1] += cell_start[c];
    cell_atoms.resize(cell_start[ncell]);
    {
        std::vector<int> fill(cell_start.begin(), cell_start.end() - 1);
        for (int a = 0; a < N; a++)  // stable: file order inside a cell
            if (cell_of[a] >= 0) cell_atoms[fill[cell_of[a]]++] = a;
    }

    // map groups in kernel order (actions after main.cpp:3286-3379).  Maps that
    // keep an hbond min/max for some receptor class go first, at most NG_MM per
    // launch, so their min/max accumulators have fixed register slots.
    std::vector<int> is_partner(std::max(nAM, 1), 0);
    if (p->separate_desolvation_maps) {
        for (int m = 0; m < nAM; m++) {
            if (p->map_is_covalent[m]) continue;
            if (m + 1 < nAM) is_partner[m + 1] = 1;
            m++;
        }
    }
    std::vector<std::array<uint8_t, 8>> act(std::max(nAM, 1));
    std::vector<int> mm_maps, plain_maps;
    for (int m = 0; m < nAM; m++) {
        const bool aff = !p->map_is_covalent[m] && !is_partner[m];
        bool mm = false;
        for (int hb = 0; hb < 8; hb++) {
            uint8_t a = ACT_PLAIN;
            if (!aff) a = ACT_SKIP;
            else if (p->map_is_hbonder[m]) {
                const int mh = p->map_hbond[m];
                if ((mh == 3 || mh == 5 || mh == 6) && (hb == 1 || hb == 2 || hb == 6)) a = ACT_SUMA;
                else if ((mh == 4 || mh == 6) && (hb == 1 || hb == 2 || hb == 6)) a = ACT_MMA;
                else if ((mh == 1 || mh == 2 || mh == 6) && (hb > 2 || hb == 6)) a = ACT_MMD;
            }
            act[m][hb] = a;
            if (hb <= 6 && (a == ACT_MMA || a == ACT_MMD)) mm = true;
        }
        (mm ? mm_maps : plain_maps).push_back(m);
    }
    pl->groups.clear();
    pl->any_cov = false;
    std::vector<uint8_t> skip_map(std::max(nAM, 1), 0);  // ACT_SKIP for every class: table column left zero
    size_t im = 0, ip = 0;
    do {
        NearGroup g;
        std::memset(&g, 0, sizeof g);
        std::vector<int> order;
        while (im < mm_maps.size() && (int)order.size() < NG_MM) order.push_back(mm_maps[im++]);
        while (ip < plain_maps.size() && (int)order.size() < NG_MAX) order.push_back(plain_maps[ip++]);
        g.ng = (int)order.size();
        g.write_special = pl->groups.empty() ? 1 : 0;
        g.has_hrow = p->disorder_h ? 1 : 0;
        g.col0 = (int)pl->groups.size() * NG_MAX;
        for (int k = 0; k < g.ng; k++) {
            const int m = order[k];
            g.out_map[k] = m;
            g.cov[k] = (uint8_t)(p->map_is_covalent[m] ? 1 : 0);
            if (g.cov[k]) pl->any_cov = true;
            for (int hb = 0; hb < 8; hb++) g.actw[hb] |= (unsigned long long)act[m][hb] << (3 * k);
            skip_map[m] = 1;
            for (int hb = 0; hb < 8; hb++) skip_map[m] &= act[m][hb] == ACT_SKIP ? 1 : 0;
            // desolvation lands on the affinity map, or on its partner when maps are separate
            const bool gets_desolv = !g.cov[k] && (p->separate_desolvation_maps ? (bool)is_partner[m] : true);
            g.sp[k] = gets_desolv ? p->map_solpar_probe[m] : 0.0;
            g.vp[k] = gets_desolv ? p->map_vol_probe[m] : 0.0;
        }
        for (int hb = 0; hb < 8; hb++) {
            bool plain = true;
            for (int k = 0; k < g.ng; k++) {
                const int a = (int)((g.actw[hb] >> (3 * k)) & 7ull);
                plain &= (a == ACT_PLAIN || a == ACT_SKIP);
            }
            if (plain) g.plain_hb |= 1u << hb;
            for (int r = 0; r < NG_MAX / 4; r++) {
                bool row_plain = true;
                for (int k = 4 * r; k < 4 * r + 4 && k < g.ng; k++) {
                    const int a = (int)((g.actw[hb] >> (3 * k)) & 7ull);
                    row_plain &= (a == ACT_PLAIN || a == ACT_SKIP);
                }
                if (row_plain) g.plain4 |= 1u << (4 * hb + r);
            }
        }
        pl->groups.push_back(g);
    } while (im < mm_maps.size() || ip < plain_maps.size());

    // tables: vdW/H-bond transposed to [type][bin][column], columns in kernel order
    pl->mpad = (int)pl->groups.size() * NG_MAX;
    const int nT = std::max(1, p->n_rec_types);
    std::vector<int> colmap(pl->mpad, -1);
    for (const NearGroup &g : pl->groups)
        for (int k = 0; k < g.ng; k++)
            if (!skip_map[g.out_map[k]]) colmap[g.col0 + k] = g.out_map[k];
    std::vector<float> vdwT, etab, solf;
    std::vector<double> reps;
    if (!dev_tables) {
        vdwT.assign((size_t)nT * AG_NEINT * pl->mpad, 0.f);
        for (int c = 0; c < pl->mpad; c++) {
            const int m = colmap[c];
            if (m < 0) continue;
            for (int t = 0; t < p->n_rec_types; t++)
                for (int b = 0; b < AG_NEINT; b++)
                    vdwT[((size_t)t * AG_NEINT + b) * pl->mpad + c] = p->e_vdw_hb[((size_t)t * nAM + m) * AG_NEINT + b];
        }
        etab.resize(AG_NDIEL);
        solf.resize(AG_NDIEL);
        reps.assign(AG_NDIEL, 0.0);
        for (int k = 0; k < AG_NDIEL; k++) {
            const double f = p->dddiel ? p->r_epsilon_fn[k] : p->invdielcal;
            if (p->dddiel) reps[k] = p->r_epsilon_fn[k];
            etab[k] = (float)(f * p->coeff_estat);
            solf[k] = (float)p->sol_fn[k];
        }
    }

    // uploads
    double *dx, *dy, *dz, *dq, *dvol, *dsol, *drv, *drv2;
    int *dtype, *dhb, *drexp, *dh, *dcs, *dca, *dmc, *dmh, *dmhb;
    uint8_t *ddis;
    double *dms, *dmv, *dsolfn, *dreps;
    AGB_CK(upload(B, "x", x.data(), N, &dx, s, acc));
    AGB_CK(upload(B, "y", y.data(), N, &dy, s, acc));
    AGB_CK(upload(B, "z", z.data(), N, &dz, s, acc));
    AGB_CK(upload(B, "q", p->charge, N, &dq, s, acc));
    AGB_CK(upload(B, "vol", p->vol, N, &dvol, s, acc));
    AGB_CK(upload(B, "solpar", p->solpar, N, &dsol, s, acc));
    AGB_CK(upload(B, "rv", p->rvector, 3 * (size_t)N, &drv, s, acc));
    AGB_CK(upload(B, "rv2", p->rvector2, 3 * (size_t)N, &drv2, s, acc));
    AGB_CK(upload(B, "type", p->rec_type, N, &dtype, s, acc));
    AGB_CK(upload(B, "hbond", p->hbond, N, &dhb, s, acc));
    AGB_CK(upload(B, "rexp", p->rexp, N, &drexp, s, acc));
    AGB_CK(upload(B, "disorder", p->disorder, N, &ddis, s, acc));
    AGB_CK(upload(B, "atomA", atomA.data(), atomA.size(), &pl->atomA, s, acc));
    AGB_CK(upload(B, "atomB", atomB.data(), atomB.size(), &pl->atomB, s, acc));
    AGB_CK(upload(B, "meta", meta.data(), meta.size(), &pl->meta, s, acc));
    AGB_CK(upload(B, "h_index", h_index.data(), h_index.size(), &dh, s, acc));
    AGB_CK(upload(B, "cell_start", cell_start.data(), cell_start.size(), &dcs, s, acc));
    AGB_CK(upload(B, "cell_atoms", cell_atoms.data(), cell_atoms.size(), &dca, s, acc));
    std::vector<int> mc(std::max(nAM, 1), 0), mh(std::max(nAM, 1), 0), mhb(std::max(nAM, 1), 0);
    std::vector<double> ms(std::max(nAM, 1), 0.0), mv(std::max(nAM, 1), 0.0);
    for (int m = 0; m < nAM; m++) {
        mc[m] = p->map_is_covalent[m]; mh[m] = p->map_is_hbonder[m]; mhb[m] = p->map_hbond[m];
        ms[m] = p->map_solpar_probe[m]; mv[m] = p->map_vol_probe[m];
    }
    AGB_CK(upload(B, "m_cov", mc.data(), mc.size(), &dmc, s, acc));
    AGB_CK(upload(B, "m_hb", mh.data(), mh.size(), &dmh, s, acc));
    AGB_CK(upload(B, "m_hbond", mhb.data(), mhb.size(), &dmhb, s, acc));
    AGB_CK(upload(B, "m_solpar", ms.data(), ms.size(), &dms, s, acc));
    AGB_CK(upload(B, "m_vol", mv.data(), mv.size(), &dmv, s, acc));
    if (!dev_tables) {
        AGB_CK(upload(B, "vdwT", vdwT.data(), vdwT.size(), &pl->vdwT, s, acc));
        AGB_CK(upload(B, "etab", etab.data(), etab.size(), &pl->etab, s, acc));
        AGB_CK(upload(B, "solf", solf.data(), solf.size(), &pl->solf, s, acc));
        AGB_CK(upload(B, "sol_fn", p->sol_fn, AG_NDIEL, &dsolfn, s, acc));
        AGB_CK(upload(B, "reps", reps.data(), reps.size(), &dreps, s, acc));
    } else {
        // tables already on the device (e.g. from ag_tables_build): packed by kernels
        int *dcol;
        void *vv;
        AGB_CK(upload(B, "colmap", colmap.data(), colmap.size(), &dcol, s, acc));
        AGB_CK(B->ensure("vdwT", (size_t)nT * AG_NEINT * pl->mpad * sizeof(float), &vv)); pl->vdwT = (float *)vv;
        AGB_CK(B->ensure("far_tab", ((size_t)pl->tab_len + AG_NDIEL) * sizeof(float), &vv)); pl->far_tab = (float *)vv;
        AGB_CK(B->ensure("etab", AG_NDIEL * sizeof(float), &vv)); pl->etab = (float *)vv;
        AGB_CK(B->ensure("solf", AG_NDIEL * sizeof(float), &vv)); pl->solf = (float *)vv;
        AGB_CK(B->ensure("sol_fn", AG_NDIEL * sizeof(double), &vv)); dsolfn = (double *)vv;
        AGB_CK(B->ensure("reps", AG_NDIEL * sizeof(double), &vv)); dreps = (double *)vv;
        AGB_CK(cudaMemcpyAsync(dsolfn, p->sol_fn, AG_NDIEL * sizeof(double), cudaMemcpyDeviceToDevice, s));
        AGB_CK(cudaMemsetAsync(pl->vdwT, 0, (size_t)nT * AG_NEINT * pl->mpad * sizeof(float), s));
        AGB_CK(launch_pack_tables(p->e_vdw_hb, p->n_rec_types, nAM, dcol, pl->mpad, pl->vdwT, p->sol_fn,
                                  p->dddiel ? p->r_epsilon_fn : nullptr, p->dddiel, p->invdielcal, p->coeff_estat,
                                  pl->far_tab, pl->tab_len, pl->etab, pl->solf, dreps, s));
    }

    d.x = dx; d.y = dy; d.z = dz; d.q = dq; d.vol = dvol; d.solpar = dsol; d.rv = drv; d.rv2 = drv2;
    d.type = dtype; d.hbond = dhb; d.rexp = drexp; d.disorder = ddis;
    d.n_h = (int)h_index.size(); d.h_index = dh;
    d.cell_start = dcs; d.cell_atoms = dca;
    d.m_cov = dmc; d.m_hb = dmh; d.m_hbond = dmhb; d.m_solpar = dms; d.m_vol = dmv;
    d.vdw = pl->vdwT; d.sol_fn = dsolfn; d.reps = dreps; d.far_tab = pl->far_tab;

    // outputs and scratch
    pl->floating = p->floating_grid ? 1 : 0;
    pl->constriction = p->constriction_grid ? 1 : 0;
    pl->constriction_cutoff = p->constriction_cutoff;
    const size_t n_out = (size_t)p->n_maps + pl->floating + pl->constriction;
    if (pl->opts.precision == AG_PREC_FP64) {
        AGB_CK(B->ensure("maps64", n_out * P * sizeof(double), &v));
        pl->maps64 = (double *)v;
        pl->maps32 = nullptr;
    } else {
        AGB_CK(B->ensure("maps32", n_out * P * sizeof(float), &v));
        pl->maps32 = (float *)v;
        pl->maps64 = nullptr;
    }
    if (pl->any_cov) {
        AGB_CK(B->ensure("cov", P * sizeof(double), &v));
        pl->cov = (double *)v;
    } else {
        pl->cov = nullptr;
    }
    if (pl->far_partial && d.elec_map >= 0) {
        const ReduceInst r{d.P, pl->n_chunks, pl->far_partial, pl->maps32 + (size_t)d.elec_map * P};
        const long long beg[2] = {0, d.P};
        AGB_CK(B->ensure("reduce", sizeof r, &v));
        pl->d_reduce = (ReduceInst *)v;
        AGB_CK(B->ensure("reduce_begin", sizeof beg, &v));
        pl->d_reduce_begin = (long long *)v;
        AGB_CK(cudaMemcpyAsync(pl->d_reduce, &r, sizeof r, cudaMemcpyHostToDevice, s));
        AGB_CK(cudaMemcpyAsync(pl->d_reduce_begin, beg, sizeof beg, cudaMemcpyHostToDevice, s));
        AGB_CK(cudaStreamSynchronize(s));  // sources are locals
    } else {
        pl->d_reduce = nullptr;
        pl->d_reduce_begin = nullptr;
    }
    return AG_OK;
}

// Bin-guard multipliers of the far kernel for a grid spacing (in bins):
// far_edge_multipliers with the largest frame-relative point coordinate and
// whether every frame point coordinate il*spacing_adiv is an exact float.
// rsqrt.approx.f32 is taken at 2.5 * 2^-24 relative error (PTX ISA:
// 2^-22.9 = 2.14 * 2^-24; checked on the device by ag_diag_rsqrt_error).
void far_guard(double spacing_adiv, float *lo, float *hi)
{
    bool exact = true;
    for (int il = 0; il < FRAME_X; il++) {
        const double v = (double)il * spacing_adiv;
        exact &= std::fma((double)il, spacing_adiv, -v) == 0.0 && (double)(float)v == v;
    }
    const double px = (FRAME_X - 1) * spacing_adiv, pyz = (FRAME_Y - 1) * spacing_adiv;
    far_edge_multipliers(std::sqrt(px * px + 2 * pyz * pyz), exact, 2.5, lo, hi);
}

FarArgs far_args(const ag_plan *pl)
{
    const DevProblem &d = pl->dp;
    FarArgs a;
    std::memset(&a, 0, sizeof a);
    a.ax128 = pl->x128; a.ay128 = pl->y128; a.az128 = pl->z128; a.qw = pl->qw;
    a.far_tab = pl->far_tab; a.partial = pl->far_partial;
    a.spacing_adiv = d.spacing * AG_A_DIV; a.P = d.P;
    a.n_atoms = d.n_atoms; a.chunk_atoms = pl->chunk_atoms;
    a.n1x = d.n1x; a.n1y = d.n1y; a.n1z = d.n1z; a.nex = d.nex; a.ney = d.ney; a.nez = d.nez;
    a.nfx = frames_x(d.n1x); a.nfy = frames_y(d.n1y); a.nfz = frames_z(d.n1z);
    a.tab_mode = pl->far_mode;
    a.tab_const = pl->far_const;
    a.tab_full = pl->far_tab ? pl->far_tab + pl->tab_len : nullptr;
    a.tab_len = pl->far_mode == FAR_TAB_CONST ? 0 : pl->tab_len;
    a.clamp = pl->far_clamp;
    far_guard(a.spacing_adiv, &a.edge_lo, &a.edge_hi);
    a.edge_bits = pl->edge_bits;
    a.edge_words = far_edge_words(pl->chunk_atoms);
    a.edge_counters = pl->ctx ? pl->ctx->d_counters + 2 : nullptr;
    return a;
}

// Kernels launched for the far field of one run: the far-field kernel, and
// the fix-up unless the table is constant (no guard bins then).
int far_launches(const FarArgs &fa) { return (fa.tab_mode != FAR_TAB_CONST && fa.edge_bits) ? 2 : 1; }

NearPtrs near_ptrs(const ag_plan *pl, unsigned long long *counters)
{
    NearPtrs q;
    q.atomA = pl->atomA; q.atomB = pl->atomB; q.meta = pl->meta; q.vdwT = pl->vdwT; q.mpad = pl->mpad;
    q.etab = pl->etab; q.solf = pl->solf; q.cov_map = pl->cov; q.out32 = pl->maps32; q.out64 = pl->maps64;
    q.counters = counters;
    return q;
}

// Far-field z-slab k of nslab on the side stream; slab 0 first forks the side
// stream from s.  far_done[k] marks the slab's end; evf0/evf1 bracket all slabs.
ag_status launch_far_slab(ag_plan *pl, cudaStream_t s, int k, int nslab)
{
    ag_context *c = pl->ctx;
    if (k == 0) {
        AGB_CK(cudaEventRecord(c->fork, s));
        AGB_CK(cudaStreamWaitEvent(c->side, c->fork, 0));
        AGB_CK(cudaEventRecord(c->evf0, c->side));
    }
    int z0, z1;
    slab_range(pl->dp, k, &z0, &z1);
    const int fz0 = z0 / FRAME_Z, fz1 = (k == nslab - 1) ? -1 : z1 / FRAME_Z;
    const FarArgs fa = far_args(pl);
    AGB_CK(launch_emap_far(fa, pl->n_chunks, 512, c->side, fz0, fz1));
    AGB_CK(launch_far_fixup(fa, pl->n_chunks, c->side, fz0, fz1));
    AGB_CK(cudaEventRecord(c->far_done[k], c->side));
    if (k == nslab - 1) AGB_CK(cudaEventRecord(c->evf1, c->side));
    return AG_OK;
}

// FP32 run as z-slabs (slab_range: whole far-field frames and near-field
// brick rows), submitted slab by slab: far slab k on the side
// stream (unless the plan launched it already); near slab k on s, then (after
// far slab k) the e-map reduction of slab k, then event red_done[k].  The far
// and near kernels of neighbouring slabs overlap, and a caller can copy slab k
// as soon as red_done[k] fires.
ag_status enqueue_slabs(ag_plan *pl, cudaStream_t s, int nslab, int &launches)
{
    const DevProblem &d = pl->dp;
    ag_context *c = pl->ctx;
    const long long plane = (long long)d.n1x * d.n1y;
    const bool far = d.elec_map >= 0 && pl->n_chunks > 0;
    const bool need_near = d.n_atom_maps > 0 || d.dsolv_map >= 0 || d.elec_map >= 0;
    for (int k = 0; k < nslab; k++) {
        if (far) {
            if (k >= pl->far_early) {
                ag_status st = launch_far_slab(pl, s, k, nslab);
                if (st != AG_OK) return st;
            }
            launches += far_launches(far_args(pl));
        }
        int sz0, sz1;
        slab_range(d, k, &sz0, &sz1);
        const int bz0 = sz0 / 4, bz1 = (k == nslab - 1) ? -1 : sz1 / 4;  // 8x8x4 bricks
        if (need_near)
            for (const NearGroup &g : pl->groups) {
                AGB_CK(launch_near(false, d, g, near_ptrs(pl, c->d_counters), 0, s, bz0, bz1));
                launches++;
            }
        if (far) {
            const long long z0 = sz0, z1 = sz1;
            const ReduceInst r{d.P, pl->n_chunks, pl->far_partial, pl->maps32 + (size_t)d.elec_map * d.P};
            AGB_CK(cudaStreamWaitEvent(s, c->far_done[k], 0));
            AGB_CK(launch_emap_reduce_range(r, z0 * plane, z1 * plane, s));
            launches++;
        }
        AGB_CK(cudaEventRecord(c->red_done[k], s));
    }
    return AG_OK;
}


// 'map_receptor_interior off': the collision rule over points [lin0, lin1),
// after the e map and the distance maps are complete.
ag_status launch_plan_collisions(ag_plan *pl, cudaStream_t s, long long lin0, long long lin1)
{
    const DevProblem &d = pl->dp;
    const size_t P = (size_t)d.P, f = (size_t)d.n_maps * P, cc = f + (size_t)pl->floating * P;
    if (pl->maps64)
        AGB_CK(launch_collisions(d, lin0, lin1, pl->constriction_cutoff, nullptr, nullptr, nullptr,
                                 d.elec_map >= 0 ? pl->maps64 + (size_t)d.elec_map * P : nullptr,
                                 pl->floating ? pl->maps64 + f : nullptr, pl->constriction ? pl->maps64 + cc : nullptr,
                                 s));
    else
        AGB_CK(launch_collisions(d, lin0, lin1, pl->constriction_cutoff,
                                 d.elec_map >= 0 ? pl->maps32 + (size_t)d.elec_map * P : nullptr,
                                 pl->floating ? pl->maps32 + f : nullptr, pl->constriction ? pl->maps32 + cc : nullptr,
                                 nullptr, nullptr, nullptr, s));
    return AG_OK;
}

// A z-slab [z0, z1) of the grid is a shard of the map set: its points need
// every atom but no other plane.  z0 is a multiple of FRAME_Z (whole far-field
// frame rows, which hold whole near-field brick rows) and z1 one too or n1z.
ag_status check_zslab(const ag_problem *p, int z0, int z1)
{
    if (!p) return invalid("null problem");
    const int n1z = p->n1[2];
    if (z0 < 0 || z1 > n1z || z0 >= z1) return invalid("z-slab outside the grid or empty");
    if (z0 % FRAME_Z != 0 || (z1 != n1z && z1 % FRAME_Z != 0))
        return invalid("z-slab bounds must be multiples of 8 planes (or the last plane)");
    return AG_OK;
}

// FP32 kernels of planes [z0, z1) only (check_zslab), on s with the far field
// on the side stream as run_plan; the maps of those planes land at their
// places in the plan's full-grid buffers.  Each point's work is the one-shot
// call's, so the planes equal it bit for bit when the plan has its chunking.
ag_status run_plan_zrange(ag_plan *pl, cudaStream_t s, int z0, int z1)
{
    ag_context *c = pl->ctx;
    const DevProblem &d = pl->dp;
    int launches = 0;
    AGB_CK(cudaMemsetAsync(c->d_counters, 0, kCounters * sizeof(unsigned long long), s));
    AGB_CK(cudaEventRecord(c->ev0, s));
    const bool far = d.elec_map >= 0 && pl->n_chunks > 0;
    const bool last = z1 == d.n1z;
    if (far) {
        AGB_CK(cudaEventRecord(c->fork, s));
        AGB_CK(cudaStreamWaitEvent(c->side, c->fork, 0));
        AGB_CK(cudaEventRecord(c->evf0, c->side));
        const FarArgs fa = far_args(pl);
        AGB_CK(launch_emap_far(fa, pl->n_chunks, 512, c->side, z0 / FRAME_Z, last ? -1 : z1 / FRAME_Z));
        AGB_CK(cudaEventRecord(c->evfx, c->side));
        AGB_CK(launch_far_fixup(fa, pl->n_chunks, c->side, z0 / FRAME_Z, last ? -1 : z1 / FRAME_Z));
        AGB_CK(cudaEventRecord(c->evf1, c->side));
        AGB_CK(cudaEventRecord(c->join, c->side));
        launches += far_launches(fa);
    }
    if (pl->any_cov) {
        AGB_CK(launch_covalent(d, pl->cov, s));
        launches++;
    }
    if (pl->floating || pl->constriction) {
        const size_t P = (size_t)d.P, f = (size_t)d.n_maps * P, cc = f + (size_t)pl->floating * P;
        AGB_CK(launch_distance_maps(d, pl->constriction_cutoff, pl->floating ? pl->maps32 + f : nullptr,
                                    pl->constriction ? pl->maps32 + cc : nullptr, nullptr, nullptr, s));
        launches++;
    }
    const bool need_near = d.n_atom_maps > 0 || d.dsolv_map >= 0 || d.elec_map >= 0;
    if (need_near)
        for (const NearGroup &g : pl->groups) {
            AGB_CK(launch_near(false, d, g, near_ptrs(pl, c->d_counters), 0, s, z0 / 4, last ? -1 : z1 / 4));
            launches++;
        }
    if (far) {
        const long long plane = (long long)d.n1x * d.n1y;
        const ReduceInst r{d.P, pl->n_chunks, pl->far_partial, pl->maps32 + (size_t)d.elec_map * d.P};
        AGB_CK(cudaStreamWaitEvent(s, c->join, 0));
        AGB_CK(launch_emap_reduce_range(r, (long long)z0 * plane, (long long)z1 * plane, s));
        launches++;
    }
    if (d.report_collisions) {
        const long long plane = (long long)d.n1x * d.n1y;
        ag_status st = launch_plan_collisions(pl, s, (long long)z0 * plane, (long long)z1 * plane);
        if (st != AG_OK) return st;
        launches++;
    }
    AGB_CK(cudaEventRecord(c->ev1, s));
    pl->last_launches = launches;
    c->pending = true;
    c->had_far = far;
    c->had_fixup_event = far;
    c->had_near = false;
    c->last_launches = launches;
    c->last_far_pairs = (d.elec_map >= 0) ? (int64_t)(z1 - z0) * d.n1x * d.n1y * d.n_atoms : 0;
    return AG_OK;
}

ag_status run_plan(ag_plan *pl, cudaStream_t s)
{
    ag_context *c = pl->ctx;
    const DevProblem &d = pl->dp;
    const bool exact = pl->opts.precision == AG_PREC_FP64;
    int launches = 0;
    AGB_CK(cudaMemsetAsync(c->d_counters, 0, kCounters * sizeof(unsigned long long), s));
    AGB_CK(cudaEventRecord(c->ev0, s));
    const bool far = !exact && d.elec_map >= 0 && pl->n_chunks > 0;
    if (d.elec_map >= 0 && exact) {
        AGB_CK(launch_emap_exact(d, pl->maps64 + (size_t)d.elec_map * d.P, s));
        launches++;
    }
    // far field on the side stream, concurrent with the near-field kernel (or,
    // with opts.serial, before it on s)
    const bool serial = pl->opts.serial != 0;
    cudaStream_t fs = serial ? s : c->side;
    if (far) {
        if (!serial) {
            AGB_CK(cudaEventRecord(c->fork, s));
            AGB_CK(cudaStreamWaitEvent(c->side, c->fork, 0));
        }
        AGB_CK(cudaEventRecord(c->evf0, fs));
        const FarArgs fa = far_args(pl);
        AGB_CK(launch_emap_far(fa, pl->n_chunks, 512, fs));
        AGB_CK(cudaEventRecord(c->evfx, fs));
        AGB_CK(launch_far_fixup(fa, pl->n_chunks, fs));
        AGB_CK(cudaEventRecord(c->evf1, fs));
        if (!serial) AGB_CK(cudaEventRecord(c->join, fs));
        launches += far_launches(fa);
    }
    if (pl->any_cov) {
        AGB_CK(launch_covalent(d, pl->cov, s));
        launches++;
    }
    if (pl->floating || pl->constriction) {
        const size_t P = (size_t)d.P, f = (size_t)d.n_maps * P, c = f + (size_t)pl->floating * P;
        if (exact)
            AGB_CK(launch_distance_maps(d, pl->constriction_cutoff, nullptr, nullptr,
                                        pl->floating ? pl->maps64 + f : nullptr,
                                        pl->constriction ? pl->maps64 + c : nullptr, s));
        else
            AGB_CK(launch_distance_maps(d, pl->constriction_cutoff, pl->floating ? pl->maps32 + f : nullptr,
                                        pl->constriction ? pl->maps32 + c : nullptr, nullptr, nullptr, s));
        launches++;
    }
    const bool need_near = d.n_atom_maps > 0 || d.dsolv_map >= 0 || (!exact && d.elec_map >= 0);
    AGB_CK(cudaEventRecord(c->evn0, s));
    if (need_near) {
        for (const NearGroup &g : pl->groups) {
            AGB_CK(launch_near(exact, d, g, near_ptrs(pl, c->d_counters), 0, s));
            launches++;
        }
    }
    AGB_CK(cudaEventRecord(c->evn1, s));
    if (far) {
        if (!serial) AGB_CK(cudaStreamWaitEvent(s, c->join, 0));
        AGB_CK(launch_emap_reduce(pl->d_reduce, pl->d_reduce_begin, 1, d.P, s));
        launches++;
    }
    if (d.report_collisions) {
        ag_status st = launch_plan_collisions(pl, s, 0, d.P);
        if (st != AG_OK) return st;
        launches++;
    }
    AGB_CK(cudaEventRecord(c->ev1, s));
    pl->last_launches = launches;
    c->pending = true;
    c->had_far = !exact && d.elec_map >= 0 && pl->n_chunks > 0;
    c->had_near = true;
    c->had_fixup_event = c->had_far;
    c->last_launches = launches;
    c->last_far_pairs = (d.elec_map >= 0) ? (int64_t)d.P * d.n_atoms : 0;
    return AG_OK;
}

ag_status settle_stats(ag_context *c)
{
    if (!c->pending) return AG_OK;
    AGB_CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f, fms = 0.f, xms = 0.f, nms = 0.f;
    AGB_CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (c->had_far) AGB_CK(cudaEventElapsedTime(&fms, c->evf0, c->evf1));
    if (c->had_far && c->had_fixup_event) AGB_CK(cudaEventElapsedTime(&xms, c->evfx, c->evf1));
    if (c->had_near) AGB_CK(cudaEventElapsedTime(&nms, c->evn0, c->evn1));
    unsigned long long h[kCounters] = {};
    AGB_CK(cudaMemcpy(h, c->d_counters, sizeof h, cudaMemcpyDeviceToHost));
    c->stats.near_pairs = (int64_t)h[0];
    c->stats.fp64_fallbacks = (int64_t)h[1];
    c->stats.far_edge_pairs = (int64_t)h[2];
    c->stats.far_fp32_bin_errors = (int64_t)h[3];
    c->stats.far_fp64_ties = (int64_t)h[4];
    c->stats.far_pairs = c->last_far_pairs;
    c->stats.gpu_launches = c->last_launches;
    c->stats.kernel_ms = ms;
    c->stats.far_ms = fms;
    c->stats.fixup_ms = xms;
    c->stats.near_ms = nms;
    c->pending = false;
    return AG_OK;
}

ag_status finish_stats(ag_plan *pl) { return settle_stats(pl->ctx); }

ag_status make_plan(ag_context *ctx, const ag_problem *p, const ag_opts *o, bool own, ag_plan **out,
                    Arena *arena = nullptr, bool pipelined = false, cudaStream_t stream = nullptr,
                    bool early_far = true);

}  // namespace

struct ag_batch {
    ag_context *ctx = nullptr;
    cudaStream_t stream = nullptr;  // uploads of the batch's set-up (the context's stream unless pipelined)
    std::unique_ptr<Arena> arena;  // declared before the plans: released after them
    std::vector<std::unique_ptr<ag_plan>> plans;
    std::vector<FarArgs> far;         // per instance, in work order
    std::vector<NearInst> near;       // per (instance, group), in work order
    std::vector<long long> far_begin, near_begin;
    BufferSet bufs;
    std::vector<ReduceInst> red;       // e-map reduction per instance with a far field
    std::vector<long long> red_begin;
    ReduceInst *d_red = nullptr;
    long long *d_red_begin = nullptr;
    FarArgs *d_far = nullptr;
    NearInst *d_near = nullptr;
    long long *d_far_begin = nullptr, *d_near_begin = nullptr;
    unsigned long long *d_counters = nullptr;  // kCounters: see its definition
    ag_tuning tune{};
    int far_ctas_per_sm = 3, near_ctas_per_sm = 3;  // resident CTAs per SM of the persistent kernels
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~ag_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace {

// Far-field work units of one instance with the given chunking.
long long far_units(const FarArgs &a) { return (long long)a.nfx * a.nfy * a.nfz * ((a.n_atoms + a.chunk_atoms - 1) / std::max(1, a.chunk_atoms)); }

ag_status batch_upload_far(ag_batch *b, bool chunked)
{
    // chunking: one unit per (frame, all atoms), or per (frame, 2048-atom chunk)
    b->far_begin.assign(1, 0);
    for (size_t i = 0; i < b->far.size(); i++) {
        FarArgs &a = b->far[i];
        a.chunk_atoms = chunked ? std::min(2048, std::max(a.n_atoms, 1)) : std::max(a.n_atoms, 1);
        a.edge_words = far_edge_words(a.chunk_atoms);
        b->far_begin.push_back(b->far_begin.back() + (a.n_atoms > 0 ? far_units(a) : 0));
    }
    // e-map reduction: each instance's partial chunks, for this chunking
    for (size_t i = 0; i < b->far.size(); i++) {
        const FarArgs &a = b->far[i];
        b->red[i].n_chunks = a.n_atoms > 0 ? (a.n_atoms + a.chunk_atoms - 1) / a.chunk_atoms : 0;
    }
    if (!b->red.empty()) {
        AGB_CK(cudaMemcpyAsync(b->d_red, b->red.data(), sizeof(ReduceInst) * b->red.size(), cudaMemcpyHostToDevice,
                               b->stream));
        AGB_CK(cudaMemcpyAsync(b->d_red_begin, b->red_begin.data(), sizeof(long long) * b->red_begin.size(),
                               cudaMemcpyHostToDevice, b->stream));
    }
    AGB_CK(cudaMemcpyAsync(b->d_far, b->far.data(), sizeof(FarArgs) * b->far.size(), cudaMemcpyHostToDevice, b->stream));
    AGB_CK(cudaMemcpyAsync(b->d_far_begin, b->far_begin.data(), sizeof(long long) * b->far_begin.size(),
                           cudaMemcpyHostToDevice, b->stream));
    AGB_CK(cudaMemcpyAsync(b->d_near, b->near.data(), sizeof(NearInst) * b->near.size(), cudaMemcpyHostToDevice,
                           b->stream));
    return AG_OK;
}

// One run of the batch on s.  concurrent: the far-field kernel runs on the
// context's side stream alongside the near-field kernel (fork/join by
// events); otherwise they run one after the other (the autotuner times each).
ag_status batch_launch(ag_batch *b, cudaStream_t s, int tile, int shape, cudaEvent_t e0, cudaEvent_t e1, cudaEvent_t e2,
                       bool concurrent)
{
    ag_context *c = b->ctx;
    const bool far = b->far_begin.back() > 0;
    AGB_CK(cudaMemsetAsync(b->d_counters, 0, kCounters * sizeof(unsigned long long), s));
    if (e0) AGB_CK(cudaEventRecord(e0, s));
    cudaStream_t fs = s;
    if (far && concurrent) {
        AGB_CK(cudaEventRecord(c->fork, s));
        AGB_CK(cudaStreamWaitEvent(c->side, c->fork, 0));
        fs = c->side;
    }
    if (far) {
        int max_tab = 0;
        for (const FarArgs &fa : b->far) max_tab = std::max(max_tab, fa.tab_len);
        AGB_CK(launch_emap_far_batch(b->d_far, b->d_far_begin, (int)b->far.size(), b->d_counters, tile,
                                     b->far_ctas_per_sm, max_tab, fs));
        AGB_CK(launch_far_fixup_batch(b->d_far, b->d_far_begin, (int)b->far.size(), b->far_begin.back(), fs));
    }
    if (far && concurrent) AGB_CK(cudaEventRecord(c->join, fs));
    if (e1) AGB_CK(cudaEventRecord(e1, s));
    if (b->near_begin.back() > 0) {
        int max_ng = 0;
        for (const NearInst &ni : b->near) max_ng = std::max(max_ng, ni.g.ng);
        AGB_CK(launch_near_batch(b->d_near, b->d_near_begin, (int)b->near.size(), b->d_counters + 1, shape,
                                 b->near_ctas_per_sm, max_ng, s));
    }
    if (far && concurrent) AGB_CK(cudaStreamWaitEvent(s, c->join, 0));
    if (!b->red.empty())
        AGB_CK(launch_emap_reduce(b->d_red, b->d_red_begin, (int)b->red.size(), b->red_begin.back(), s));
    if (e2) AGB_CK(cudaEventRecord(e2, s));
    return AG_OK;
}

// Near work units (bricks) of every instance-group for one brick shape.
ag_status batch_set_near_shape(ag_batch *b, int shape)
{
    b->near_begin.assign(1, 0);
    for (const NearInst &ni : b->near) b->near_begin.push_back(b->near_begin.back() + near_bricks(ni.p, shape));
    AGB_CK(cudaMemcpyAsync(b->d_near_begin, b->near_begin.data(), sizeof(long long) * b->near_begin.size(),
                           cudaMemcpyHostToDevice, b->stream));
    return AG_OK;
}

// Time one configuration (best of two runs).
ag_status batch_time(ag_batch *b, int tile, int shape, double *far_ms, double *near_ms)
{
    cudaStream_t s = b->ctx->stream;
    cudaEvent_t e[3];
    for (auto &x : e) AGB_CK(cudaEventCreate(&x));
    double bf = 1e30, bn = 1e30;
    ag_status st = AG_OK;
    for (int rep = 0; rep < 2 && st == AG_OK; rep++) {
        st = batch_launch(b, s, tile, shape, e[0], e[1], e[2], false);
        if (st != AG_OK) break;
        cudaError_t ce = cudaEventSynchronize(e[2]);
        if (ce != cudaSuccess) { st = cuda_fail(ce, "cudaEventSynchronize"); break; }
        float f = 0, n = 0;
        cudaEventElapsedTime(&f, e[0], e[1]);
        cudaEventElapsedTime(&n, e[1], e[2]);
        bf = std::min(bf, (double)f);
        bn = std::min(bn, (double)n);
    }
    for (auto &x : e) cudaEventDestroy(x);
    *far_ms = bf;
    *near_ms = bn;
    return st;
}

// The autotuner: far tile x chunking, then near brick shape, on this batch.
ag_status batch_autotune(ag_batch *b)
{
    ag_tuning &t = b->tune;
    t = ag_tuning{};
    double best_far = 1e30, best_near = 1e30;
    int best_tile = 512, best_chunked = 0, best_shape = 0;
    const int tiles[3] = {512, 256, 1024};
    for (int chunked = 0; chunked < 2; chunked++) {
        ag_status st = batch_upload_far(b, chunked != 0);
        if (st != AG_OK) return st;
        for (int ti = 0; ti < 3; ti++) {
            double f = 0, n = 0;
            st = batch_time(b, tiles[ti], 0, &f, &n);
            if (st != AG_OK) return st;
            t.candidates++;
            if (chunked == 0 && ti == 0) { t.far_ms_default = f; t.near_ms_default = n; }
            if (f < best_far) { best_far = f; best_tile = tiles[ti]; best_chunked = chunked; }
        }
    }
    ag_status st = batch_upload_far(b, best_chunked != 0);
    if (st != AG_OK) return st;
    for (int shape = 0; shape < 3; shape++) {
        double f = 0, n = 0;
        st = batch_set_near_shape(b, shape);
        if (st != AG_OK) return st;
        st = batch_time(b, best_tile, shape, &f, &n);
        if (st != AG_OK) return st;
        t.candidates++;
        if (n < best_near) { best_near = n; best_shape = shape; }
    }
    t.far_tile = best_tile;
    t.far_chunked = best_chunked;
    t.near_shape = best_shape;
    t.far_ms = best_far;
    t.near_ms = best_near;
    return AG_OK;
}

ag_status make_plan(ag_context *ctx, const ag_problem *p, const ag_opts *o, bool own, ag_plan **out, Arena *arena,
                    bool pipelined, cudaStream_t stream, bool early_far)
{
    if (!ctx || !p || !out) return invalid("null argument");
    ag_opts opts{};
    if (o) opts = *o;
    if (opts.precision != AG_PREC_FP32 && opts.precision != AG_PREC_FP64) return invalid("unknown precision");
    if (opts.table_mode != AG_TABLE_NEAREST) {
        set_last_error("the drop-in path reads nearest-bin tables; linear tables are the differentiable mode (ag_diff_create)");
        return AG_ERR_UNSUPPORTED;
    }
    AGB_CK(cudaSetDevice(ctx->device));
    std::unique_ptr<ag_plan> pl(new ag_plan());
    pl->ctx = ctx;
    pl->opts = opts;
    if (own) {
        pl->own.reset(new BufferSet());
        pl->own->arena = arena;
        pl->bufs = pl->own.get();
    } else {
        pl->bufs = &ctx->pool;
    }
    ag_status st = build_plan(pl.get(), p, stream ? stream : ctx->stream, pipelined, early_far);
    if (st != AG_OK) return st;
    *out = pl.release();
    return AG_OK;
}

}  // namespace

extern "C" {

ag_status ag_context_create(int32_t device, ag_context **out)
{
    if (!out) return invalid("null argument");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_last_error(std::string("no CUDA device: ") + (e == cudaSuccess ? "count is 0" : cudaGetErrorString(e)));
        return AG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return invalid("device index out of range");
    std::unique_ptr<ag_context> c(new ag_context());
    c->device = device;
    AGB_CK(cudaSetDevice(device));
    AGB_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    AGB_CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    AGB_CK(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    AGB_CK(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming));
    AGB_CK(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking));
    AGB_CK(cudaEventCreateWithFlags(&c->copy_done, cudaEventDisableTiming));
    c->far_done.resize(kMaxSlabs);
    c->red_done.resize(kMaxSlabs);
    for (int k = 0; k < kMaxSlabs; k++) {
        AGB_CK(cudaEventCreateWithFlags(&c->far_done[k], cudaEventDisableTiming));
        AGB_CK(cudaEventCreateWithFlags(&c->red_done[k], cudaEventDisableTiming));
    }
    AGB_CK(cudaEventCreate(&c->ev0));
    AGB_CK(cudaEventCreate(&c->ev1));
    AGB_CK(cudaEventCreate(&c->evf0));
    AGB_CK(cudaEventCreate(&c->evf1));
    AGB_CK(cudaEventCreate(&c->evfx));
    AGB_CK(cudaEventCreate(&c->evn0));
    AGB_CK(cudaEventCreate(&c->evn1));
    AGB_CK(cudaMalloc(&c->d_counters, kCounters * sizeof(unsigned long long)));
    AGB_CK(cudaMemset(c->d_counters, 0, kCounters * sizeof(unsigned long long)));
    for (cudaEvent_t &e : c->tev) AGB_CK(cudaEventCreate(&e));
    // shared-memory limits of the far kernels on this device, set here (once
    // per context, outside any stream capture) rather than at launch
    AGB_CK(prepare_far_kernels());
    AGB_CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    *out = c.release();
    return AG_OK;
}

ag_status ag_context_cached_bytes(ag_context *ctx, int64_t *bytes)
{
    if (!ctx || !bytes) return invalid("null argument");
    *bytes = (int64_t)ctx->blocks.bytes();
    return AG_OK;
}

ag_status ag_context_trim(ag_context *ctx, int64_t *released)
{
    if (!ctx) return invalid("null context");
    DeviceGuard dg(ctx->device);
    // blocks in the cache belong to no live batch; work still queued on the
    // context's streams may use blocks of live batches only
    const size_t n = ctx->blocks.release();
    if (released) *released = (int64_t)n;
    return AG_OK;
}

ag_status ag_context_destroy(ag_context *ctx)
{
    if (!ctx) return AG_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    if (ctx->copy) cudaStreamSynchronize(ctx->copy);
    for (cudaEvent_t e : ctx->far_done) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->red_done) cudaEventDestroy(e);
    if (ctx->copy_done) cudaEventDestroy(ctx->copy_done);
    if (ctx->copy) cudaStreamDestroy(ctx->copy);
    if (ctx->d_counters) cudaFree(ctx->d_counters);
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->join) cudaEventDestroy(ctx->join);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->evf0) cudaEventDestroy(ctx->evf0);
    if (ctx->evf1) cudaEventDestroy(ctx->evf1);
    if (ctx->evfx) cudaEventDestroy(ctx->evfx);
    if (ctx->evn0) cudaEventDestroy(ctx->evn0);
    if (ctx->evn1) cudaEventDestroy(ctx->evn1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->h_text) cudaFreeHost(ctx->h_text);
    for (cudaEvent_t e : ctx->tev)
        if (e) cudaEventDestroy(e);
    delete ctx;
    return AG_OK;
}

ag_status ag_context_stats(const ag_context *ctx, ag_stats *out)
{
    if (!ctx || !out) return invalid("null argument");
    ag_status st = settle_stats(const_cast<ag_context *>(ctx));
    if (st != AG_OK) return st;
    *out = ctx->stats;
    return AG_OK;
}

// One-shot FP32 run with the maps copied to `out` slab by slab on the copy
// stream while later slabs compute.  All kernels are enqueued before the
// copies, so a pageable destination (whose copies block the host) does not
// delay the launches.
static ag_status run_plan_pipelined(ag_plan *pl, void *out, size_t n_out)
{
    ag_context *c = pl->ctx;
    const DevProblem &d = pl->dp;
    cudaStream_t s = c->stream;
    const int nslab = slab_count(d);
    const long long plane = (long long)d.n1x * d.n1y;
    int launches = 0;
    if (pl->far_early == 0) {  // else the plan cleared them and started the clock
        AGB_CK(cudaMemsetAsync(c->d_counters, 0, kCounters * sizeof(unsigned long long), s));
        AGB_CK(cudaEventRecord(c->ev0, s));
    }
    if (pl->any_cov) {
        AGB_CK(launch_covalent(d, pl->cov, s));
        launches++;
    }
    if (pl->floating || pl->constriction) {
        const size_t P = (size_t)d.P, f = (size_t)d.n_maps * P, cc = f + (size_t)pl->floating * P;
        AGB_CK(launch_distance_maps(d, pl->constriction_cutoff, pl->floating ? pl->maps32 + f : nullptr,
                                    pl->constriction ? pl->maps32 + cc : nullptr, nullptr, nullptr, s));
        launches++;
    }
    ag_status st = enqueue_slabs(pl, s, nslab, launches);
    if (st != AG_OK) return st;
    AGB_CK(cudaEventRecord(c->ev1, s));
    const bool far = d.elec_map >= 0 && pl->n_chunks > 0;
    pl->last_launches = launches;
    c->pending = true;
    c->had_far = far;
    c->had_fixup_event = false;
    c->had_near = false;
    c->last_launches = launches;
    c->last_far_pairs = (d.elec_map >= 0) ? (int64_t)d.P * d.n_atoms : 0;
    for (int k = 0; k < nslab; k++) {
        int sz0, sz1;
        slab_range(d, k, &sz0, &sz1);
        const long long z0 = sz0, z1 = sz1;
        const size_t off = (size_t)(z0 * plane) * sizeof(float), width = (size_t)((z1 - z0) * plane) * sizeof(float);
        AGB_CK(cudaStreamWaitEvent(c->copy, c->red_done[k], 0));
        AGB_CK(cudaMemcpy2DAsync((char *)out + off, (size_t)d.P * sizeof(float), (const char *)pl->maps32 + off,
                                 (size_t)d.P * sizeof(float), width, n_out, cudaMemcpyDefault, c->copy));
    }
    AGB_CK(cudaStreamSynchronize(c->copy));
    return AG_OK;
}

static ag_status compute_common(ag_context *ctx, const ag_problem *problem, const ag_opts *opts, void *maps,
                                size_t elem)
{
    if (!maps) return invalid("null maps");
    ag_plan *pl = nullptr;
    // the collision rule rewrites finished planes: one-shot calls with it do not pipeline copies
    const bool pipelined = elem == 4 && problem && problem->n1[2] > kSlabZ && !(opts && opts->serial) &&
                           !problem->report_collisions;
    ag_status st = make_plan(ctx, problem, opts, false, &pl, nullptr, pipelined);
    if (st != AG_OK) return st;
    std::unique_ptr<ag_plan> guard(pl);
    const size_t n_out = (size_t)problem->n_maps + pl->floating + pl->constriction;
    if (pipelined) {
        st = run_plan_pipelined(pl, maps, n_out);
        if (st != AG_OK) return st;
        AGB_CK(cudaStreamSynchronize(ctx->stream));
        return finish_stats(pl);
    }
    st = run_plan(pl, ctx->stream);
    if (st != AG_OK) return st;
    const void *src = elem == 8 ? (const void *)pl->maps64 : (const void *)pl->maps32;
    AGB_CK(cudaMemcpyAsync(maps, src, n_out * (size_t)pl->dp.P * elem, cudaMemcpyDefault, ctx->stream));
    AGB_CK(cudaStreamSynchronize(ctx->stream));
    return finish_stats(pl);
}

ag_status ag_maps_compute(ag_context *ctx, const ag_problem *problem, const ag_opts *opts, float *maps)
{
    if (opts && opts->precision != AG_PREC_FP32) return invalid("ag_maps_compute needs AG_PREC_FP32");
    return compute_common(ctx, problem, opts, maps, 4);
}

ag_status ag_maps_compute_f64(ag_context *ctx, const ag_problem *problem, const ag_opts *opts, double *maps)
{
    if (!opts || opts->precision != AG_PREC_FP64) return invalid("ag_maps_compute_f64 needs AG_PREC_FP64");
    return compute_common(ctx, problem, opts, maps, 8);
}

ag_status ag_maps_compute_zslab(ag_context *ctx, const ag_problem *problem, const ag_opts *opts, int32_t z0,
                                int32_t z1, float *maps)
{
    if (!maps) return invalid("null maps");
    if (opts && opts->precision != AG_PREC_FP32) return invalid("ag_maps_compute_zslab runs the FP32 path");
    ag_status st = check_zslab(problem, z0, z1);
    if (st != AG_OK) return st;
    if (!ctx) return invalid("null context");
    DeviceGuard dg(ctx->device);
    AGB_CK(dg.err);
    ag_plan *pl = nullptr;
    // the one-shot call's far-field chunking (bit-identical planes), no early launch
    st = make_plan(ctx, problem, opts, false, &pl, nullptr, problem->n1[2] > kSlabZ && !problem->report_collisions,
                   nullptr, false);
    if (st != AG_OK) return st;
    std::unique_ptr<ag_plan> guard(pl);
    st = run_plan_zrange(pl, ctx->stream, z0, z1);
    if (st != AG_OK) return st;
    const DevProblem &d = pl->dp;
    const size_t n_out = (size_t)problem->n_maps + pl->floating + pl->constriction;
    const size_t plane = (size_t)d.n1x * d.n1y, rows = (size_t)(z1 - z0) * plane;
    AGB_CK(cudaMemcpy2DAsync(maps, rows * sizeof(float), pl->maps32 + (size_t)z0 * plane, (size_t)d.P * sizeof(float),
                             rows * sizeof(float), n_out, cudaMemcpyDefault, ctx->stream));
    AGB_CK(cudaStreamSynchronize(ctx->stream));
    return finish_stats(pl);
}


ag_status ag_plan_create(ag_context *ctx, const ag_problem *problem, const ag_opts *opts, ag_plan **out)
{
    ag_opts o{};
    if (opts) o = *opts;
    if (o.precision != AG_PREC_FP32) return invalid("plans run the FP32 path; use ag_maps_compute_f64 for FP64");
    ag_status st = make_plan(ctx, problem, &o, true, out);
    if (st != AG_OK) return st;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    return AG_OK;
}

// Far-field bins of listed points against every atom (autogrid_b200_diag.h).
static ag_status far_bins_diag(ag_context *ctx, const ag_problem *problem, int32_t n_points, const int64_t *points,
                               int32_t *bin_used, int32_t *bin_fp32, int32_t *flags)
{
    if (!ctx || !problem || (n_points > 0 && (!points || !bin_used || !bin_fp32 || !flags)))
        return invalid("null argument");
    if (n_points < 0) return invalid("negative point count");
    const long long n = (long long)n_points * std::max(problem->n_atoms, 0);
    if (n > (1LL << 27)) {
        set_last_error("ag_diag_far_bins: at most 2^27 (point, atom) pairs per call");
        return AG_ERR_TOO_LARGE;
    }
    const long long P = (long long)problem->n1[0] * problem->n1[1] * problem->n1[2];
    for (int32_t i = 0; i < n_points; i++)
        if (points[i] < 0 || points[i] >= P) return invalid("point index outside the grid");
    ag_opts o{};
    ag_plan *pl = nullptr;
    ag_status st = make_plan(ctx, problem, &o, true, &pl);
    if (st != AG_OK) return st;
    std::unique_ptr<ag_plan> hold(pl);
    if (n == 0) return AG_OK;
    if (pl->far_mode != FAR_TAB_TABLE || !pl->far_tab) {
        set_last_error("ag_diag_far_bins: the problem has no far-field table (constant dielectric or no e map)");
        return AG_ERR_UNSUPPORTED;
    }
    cudaStream_t s = ctx->stream;
    long long *dpts = nullptr;
    int *dout = nullptr;
    AGB_CK(cudaMalloc(&dpts, sizeof(long long) * n_points));
    std::unique_ptr<long long, decltype(&cudaFree)> g1(dpts, &cudaFree);
    AGB_CK(cudaMalloc(&dout, sizeof(int) * 3 * (size_t)n));
    std::unique_ptr<int, decltype(&cudaFree)> g2(dout, &cudaFree);
    AGB_CK(cudaMemcpyAsync(dpts, points, sizeof(long long) * n_points, cudaMemcpyHostToDevice, s));
    FarArgs a = far_args(pl);
    a.edge_counters = nullptr;
    AGB_CK(launch_far_bins_debug(a, dpts, n_points, dout, dout + n, dout + 2 * n, s));
    AGB_CK(cudaMemcpyAsync(bin_used, dout, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
    AGB_CK(cudaMemcpyAsync(bin_fp32, dout + n, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
    AGB_CK(cudaMemcpyAsync(flags, dout + 2 * n, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
    AGB_CK(cudaStreamSynchronize(s));
    return AG_OK;
}

int ag_diag_far_bins(ag_context *ctx, const ag_problem *problem, int32_t n_points, const int64_t *points,
                     int32_t *bin_used, int32_t *bin_fp32, int32_t *flags)
{
    return (int)far_bins_diag(ctx, problem, n_points, points, bin_used, bin_fp32, flags);
}

ag_status ag_plan_run(ag_plan *plan, void *stream)
{
    if (!plan) return invalid("null plan");
    cudaStream_t s = stream ? (cudaStream_t)stream : plan->ctx->stream;
    return run_plan(plan, s);
}

ag_status ag_plan_run_zslab(ag_plan *plan, int32_t z0, int32_t z1, void *stream)
{
    if (!plan) return invalid("null plan");
    const DevProblem &d = plan->dp;
    if (z0 < 0 || z1 > d.n1z || z0 >= z1) return invalid("z-slab outside the grid or empty");
    if (z0 % FRAME_Z != 0 || (z1 != d.n1z && z1 % FRAME_Z != 0))
        return invalid("z-slab bounds must be multiples of 8 planes (or the last plane)");
    DeviceGuard dg(plan->ctx->device);
    AGB_CK(dg.err);
    return run_plan_zrange(plan, stream ? (cudaStream_t)stream : plan->ctx->stream, z0, z1);
}

const float *ag_plan_device_maps(const ag_plan *plan) { return plan ? plan->maps32 : nullptr; }

size_t ag_plan_points(const ag_plan *plan) { return plan ? (size_t)plan->dp.P : 0; }

ag_status ag_plan_download(ag_plan *plan, float *host_maps)
{
    if (!plan || !host_maps) return invalid("null argument");
    ag_context *c = plan->ctx;
    AGB_CK(cudaMemcpyAsync(host_maps, plan->maps32,
                           ((size_t)plan->dp.n_maps + plan->floating + plan->constriction) * (size_t)plan->dp.P * sizeof(float),
                           cudaMemcpyDefault, c->stream));
    AGB_CK(cudaStreamSynchronize(c->stream));
    return finish_stats(plan);
}

// Map-file text of device-resident maps (kernels/maptext.cu): measure pass,
// one small read-back of the byte counts, write pass, one copy of the text.
static ag_status format_maps(ag_context *c, const ag_problem *p, const void *dmaps, int elem, const char **text,
                             size_t *map_bytes, double *emin, double *emax)
{
    if (!c || !p || !dmaps || !text || !map_bytes) return invalid("null argument");
    if (elem != 4 && elem != 8) return invalid("elem_size must be 4 (FP32 maps) or 8 (FP64 maps)");
    if (!device_accessible(dmaps, c->device)) return invalid("ag_maps_format: the maps must be device memory of the context's GPU");
    ag_status st = validate(p);
    if (st != AG_OK) return st;
    AGB_CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const long long P = (long long)p->n1[0] * p->n1[1] * p->n1[2];
    const int n_out = p->n_maps + (p->floating_grid ? 1 : 0) + (p->constriction_grid ? 1 : 0);
    TextArgs a{};
    a.m32 = elem == 4 ? (const float *)dmaps : nullptr;
    a.m64 = elem == 8 ? (const double *)dmaps : nullptr;
    a.P = P;
    a.n_out = n_out;
    a.n_energy = p->n_maps;
    a.floating = p->floating_grid ? 1 : 0;
    a.bpm = text_blocks_per_map(P);
    const long long nb = (long long)n_out * a.bpm;
    if (nb > 0x7fffffffll) {
        set_last_error("ag_maps_format: too many grid points for one call");
        return AG_ERR_TOO_LARGE;
    }
    BufferSet &B = c->text_bufs;
    void *v;
    AGB_CK(B.ensure("len8", (size_t)nb * (size_t)text_values_per_block(), &v));
    a.len8 = (unsigned char *)v;
    AGB_CK(B.ensure("blk_len", (size_t)nb * sizeof(unsigned), &v));
    a.blk_len = (unsigned *)v;
    AGB_CK(B.ensure("blk_off", (size_t)nb * sizeof(unsigned long long), &v));
    a.blk_off = (unsigned long long *)v;
    AGB_CK(B.ensure("ext", (size_t)std::max(1, 2 * p->n_maps) * sizeof(unsigned long long), &v));
    a.ext = (unsigned long long *)v;
    AGB_CK(B.ensure("map_bytes", (size_t)(n_out + 1) * sizeof(unsigned long long), &v));
    a.map_bytes = (unsigned long long *)v;
    AGB_CK(cudaEventRecord(c->tev[0], s));
    AGB_CK(launch_text_measure(a, s));
    AGB_CK(cudaEventRecord(c->tev[1], s));
    std::vector<unsigned long long> hb((size_t)n_out + 1), he((size_t)std::max(1, 2 * p->n_maps));
    AGB_CK(cudaMemcpyAsync(hb.data(), a.map_bytes, hb.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    AGB_CK(cudaMemcpyAsync(he.data(), a.ext, he.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    AGB_CK(cudaStreamSynchronize(s));
    const size_t total = (size_t)hb[(size_t)n_out];
    AGB_CK(B.ensure("text", total, &v));
    a.text = (char *)v;
    AGB_CK(cudaEventRecord(c->tev[2], s));
    AGB_CK(launch_text_write(a, s));
    AGB_CK(cudaEventRecord(c->tev[3], s));
    if (c->h_text_cap < total || !c->h_text) {
        if (c->h_text) cudaFreeHost(c->h_text);
        c->h_text = nullptr;
        c->h_text_cap = 0;
        AGB_CK(cudaHostAlloc((void **)&c->h_text, std::max<size_t>(total, 16), cudaHostAllocDefault));
        c->h_text_cap = std::max<size_t>(total, 16);
    }
    AGB_CK(cudaMemcpyAsync(c->h_text, a.text, total, cudaMemcpyDeviceToHost, s));
    AGB_CK(cudaStreamSynchronize(s));
    float t_measure = 0.f, t_write = 0.f;
    AGB_CK(cudaEventElapsedTime(&t_measure, c->tev[0], c->tev[1]));
    AGB_CK(cudaEventElapsedTime(&t_write, c->tev[2], c->tev[3]));
    c->stats.text_ms = (double)t_measure + (double)t_write;
    c->stats.text_bytes = (int64_t)total;
    *text = c->h_text;
    for (int k = 0; k < n_out; k++) map_bytes[k] = (size_t)hb[(size_t)k];
    for (int k = 0; k < p->n_maps; k++) {
        if (emin) emin[k] = text_key_to_double(he[2 * (size_t)k]);
        if (emax) emax[k] = text_key_to_double(he[2 * (size_t)k + 1]);
    }
    return AG_OK;
}

ag_status ag_tables_build(ag_context *ctx, const ag_table_params *tp, float *e_vdw_hb, double *sol_fn,
                          double *r_epsilon_fn)
{
    if (!ctx || !tp || !e_vdw_hb || !sol_fn || (tp->dddiel && !r_epsilon_fn)) return invalid("null argument");
    const int nT = tp->n_rec_types, nAM = tp->n_atom_maps;
    if (nT < 0 || nT > AG_MAX_REC_TYPES || nAM < 0 || nAM > AG_MAX_MAPS) return invalid("table sizes out of range");
    if (nT * nAM > 0 && (!tp->cA || !tp->cB || !tp->Rij || !tp->epsij || !tp->xA || !tp->xB || !tp->map_is_covalent))
        return invalid("null parameter array");
    AGB_CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    BufferSet &B = ctx->table_bufs;
    const size_t np = (size_t)std::max(1, nT * nAM), nv = np * AG_NEINT;
    TableArgs a{};
    a.n_rec_types = nT;
    a.n_atom_maps = nAM;
    a.i_smooth = (int)(tp->r_smooth * AG_A_DIV / 2.);  // main.cpp:2190
    a.coeff_desolv = tp->coeff_desolv;
    const size_t npar = (size_t)nT * nAM;
    double *dcA, *dcB, *dR, *dE;
    int *dxA, *dxB, *dcov, *dbad;
    AGB_CK(upload(&B, "cA", tp->cA, npar, &dcA, s, nullptr));
    AGB_CK(upload(&B, "cB", tp->cB, npar, &dcB, s, nullptr));
    AGB_CK(upload(&B, "Rij", tp->Rij, npar, &dR, s, nullptr));
    AGB_CK(upload(&B, "epsij", tp->epsij, npar, &dE, s, nullptr));
    AGB_CK(upload(&B, "xA", tp->xA, npar, &dxA, s, nullptr));
    AGB_CK(upload(&B, "xB", tp->xB, npar, &dxB, s, nullptr));
    AGB_CK(upload(&B, "cov", tp->map_is_covalent, (size_t)nAM, &dcov, s, nullptr));
    a.cA = dcA; a.cB = dcB; a.Rij = dR; a.epsij = dE; a.xA = dxA; a.xB = dxB; a.map_is_covalent = dcov;
    void *v;
    AGB_CK(B.ensure("bad", sizeof(int), &v)); dbad = (int *)v;
    AGB_CK(B.ensure("raw", nv * sizeof(float), &v)); float *raw = (float *)v;
    AGB_CK(B.ensure("vdw", nv * sizeof(float), &v)); float *vdw = (float *)v;
    AGB_CK(B.ensure("sol", AG_NDIEL * sizeof(double), &v)); double *sol = (double *)v;
    AGB_CK(B.ensure("eps", AG_NDIEL * sizeof(double), &v)); double *eps = (double *)v;
    AGB_CK(cudaMemsetAsync(dbad, 0, sizeof(int), s));
    AGB_CK(cudaEventRecord(ctx->tev[0], s));
    AGB_CK(launch_tables_build(a, raw, vdw, sol, tp->dddiel ? eps : nullptr, dbad, s));
    AGB_CK(cudaEventRecord(ctx->tev[1], s));
    int bad = 0;
    AGB_CK(cudaMemcpyAsync(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost, s));
    AGB_CK(cudaStreamSynchronize(s));
    if (bad) {
        set_last_error("Van der Waals coefficient is not a number, or an exponent is 0.  AutoGrid must exit.");
        return AG_ERR_FATAL_INPUT;
    }
    if (npar) AGB_CK(cudaMemcpyAsync(e_vdw_hb, vdw, npar * AG_NEINT * sizeof(float), cudaMemcpyDefault, s));
    AGB_CK(cudaMemcpyAsync(sol_fn, sol, AG_NDIEL * sizeof(double), cudaMemcpyDefault, s));
    if (tp->dddiel) AGB_CK(cudaMemcpyAsync(r_epsilon_fn, eps, AG_NDIEL * sizeof(double), cudaMemcpyDefault, s));
    AGB_CK(cudaStreamSynchronize(s));
    float ms = 0.f;
    AGB_CK(cudaEventElapsedTime(&ms, ctx->tev[0], ctx->tev[1]));
    ctx->stats.table_ms = ms;
    return AG_OK;
}

ag_status ag_maps_format(ag_context *ctx, const ag_problem *problem, const void *device_maps, int32_t elem_size,
                         const char **text, size_t *map_bytes, double *emin, double *emax)
{
    return format_maps(ctx, problem, device_maps, elem_size, text, map_bytes, emin, emax);
}

ag_status ag_maps_compute_text(ag_context *ctx, const ag_problem *problem, const ag_opts *opts, const char **text,
                               size_t *map_bytes, double *emin, double *emax)
{
    if (!text || !map_bytes) return invalid("null argument");
    ag_plan *pl = nullptr;
    ag_status st = make_plan(ctx, problem, opts, false, &pl, nullptr, false);
    if (st != AG_OK) return st;
    std::unique_ptr<ag_plan> guard(pl);
    st = run_plan(pl, ctx->stream);
    if (st != AG_OK) return st;
    const bool f64 = pl->opts.precision == AG_PREC_FP64;
    st = format_maps(ctx, problem, f64 ? (const void *)pl->maps64 : (const void *)pl->maps32, f64 ? 8 : 4, text,
                     map_bytes, emin, emax);
    if (st != AG_OK) return st;
    return finish_stats(pl);
}

ag_status ag_plan_destroy(ag_plan *plan)
{
    if (!plan) return AG_OK;
    cudaSetDevice(plan->ctx->device);
    cudaStreamSynchronize(plan->ctx->stream);
    delete plan;
    return AG_OK;
}


// A batch whose set-up uploads go on stream `us` (the caller synchronises
// nothing else: kernels already running on the context's stream go on).
static ag_status batch_create(ag_context *ctx, const ag_problem *const *problems, int32_t n, const ag_opts *opts,
                              cudaStream_t us, ag_batch **out)
{
    if (!ctx || !problems || !out || n < 1) return invalid("ag_batch_create: bad argument");
    *out = nullptr;
    ag_opts o{};
    if (opts) o = *opts;
    if (o.precision != AG_PREC_FP32) return invalid("batches run the FP32 path");
    for (int i = 0; i < n; i++)
        if (problems[i] && problems[i]->report_collisions) {
            set_last_error("instance " + std::to_string(i) + ": batches do not report collisions "
                           "(map_receptor_interior off); use ag_maps_compute");
            return AG_ERR_UNSUPPORTED;
        }
    AGB_CK(cudaSetDevice(ctx->device));
    std::unique_ptr<ag_batch> b(new ag_batch());
    b->ctx = ctx;
    b->stream = us;
    b->arena.reset(new Arena(&ctx->blocks));
    // Instance plans (validation, cell lists, packed atoms, tables, uploads)
    // are built by a pool of host threads; device buffers come from the arena.
    b->plans.resize(n);
    std::vector<ag_status> sts(n, AG_OK);
    std::vector<std::string> errs(n);
    std::atomic<int> next{0};
    auto worker = [&]() {
        if (cudaSetDevice(ctx->device) != cudaSuccess) return;
        for (int i; (i = next.fetch_add(1)) < n;) {
            ag_plan *pl = nullptr;
            sts[i] = make_plan(ctx, problems[i], &o, true, &pl, b->arena.get(), false, us);
            if (sts[i] != AG_OK) errs[i] = ag_last_error();
            b->plans[i].reset(pl);
        }
    };
    const int nthreads = std::max(1, std::min({n, 16, (int)std::thread::hardware_concurrency()}));
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; t++) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
    for (int i = 0; i < n; i++)
        if (sts[i] != AG_OK || !b->plans[i]) {
            set_last_error("instance " + std::to_string(i) + ": " + errs[i]);
            return sts[i] != AG_OK ? sts[i] : AG_ERR_CUDA;
        }
    // work order: instances by decreasing far work (largest units first)
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const DevProblem &a = b->plans[x]->dp, &c = b->plans[y]->dp;
        return (double)a.P * (a.n_atoms + 64) > (double)c.P * (c.n_atoms + 64);
    });
    b->near_begin.assign(1, 0);
    b->red_begin.assign(1, 0);
    for (int i : order) {
        ag_plan *pl = b->plans[i].get();
        // each instance's partial buffer must hold the chunked layout (at most ceil(N/2048) chunks)
        const int max_chunks = std::max(1, (pl->dp.n_atoms + 2047) / 2048);
        if (pl->dp.elec_map >= 0 && pl->dp.n_atoms > 0) {
            void *v = nullptr;
            AGB_CK(pl->bufs->ensure("far_partial", (size_t)max_chunks * (size_t)pl->dp.P * sizeof(float), &v));
            pl->far_partial = (float *)v;
            if (pl->far_mode != FAR_TAB_CONST) {
                // edge bits for either chunking of batch_upload_far (2048-atom chunks or all atoms)
                const int nframes = frames_x(pl->dp.n1x) * frames_y(pl->dp.n1y) * frames_z(pl->dp.n1z);
                const int na = std::max(pl->dp.n_atoms, 1);
                const size_t eb = std::max(far_edge_bits_bytes(max_chunks, std::min(2048, na), nframes),
                                           far_edge_bits_bytes(1, na, nframes));
                AGB_CK(pl->bufs->ensure("edge_bits", eb, &v));
                pl->edge_bits = (uint32_t *)v;
            }
            b->far.push_back(far_args(pl));
            b->red.push_back(ReduceInst{pl->dp.P, 0, pl->far_partial, pl->maps32 + (size_t)pl->dp.elec_map * pl->dp.P});
            b->red_begin.push_back(b->red_begin.back() + pl->dp.P);
        }
        const bool need_near = pl->dp.n_atom_maps > 0 || pl->dp.dsolv_map >= 0 || pl->dp.elec_map >= 0;
        if (need_near)
            for (const NearGroup &g : pl->groups) {
                NearInst ni;
                std::memset(&ni, 0, sizeof ni);
                ni.p = pl->dp;
                ni.g = g;
                ni.ptr = near_ptrs(pl, nullptr);
                b->near.push_back(ni);
                b->near_begin.push_back(b->near_begin.back() + near_bricks(pl->dp, 0));
            }
        if (pl->any_cov) {
            AGB_CK(launch_covalent(pl->dp, pl->cov, us));  // geometry only: computed once
        }
        if (pl->floating || pl->constriction) {
            // the floating and constriction grids depend on the geometry only:
            // computed once, after the instance's energy maps (main.cpp:2958-2966)
            const size_t P = (size_t)pl->dp.P, f = (size_t)pl->dp.n_maps * P, c = f + (size_t)pl->floating * P;
            AGB_CK(launch_distance_maps(pl->dp, pl->constriction_cutoff, pl->floating ? pl->maps32 + f : nullptr,
                                        pl->constriction ? pl->maps32 + c : nullptr, nullptr, nullptr, us));
        }
    }
    void *v = nullptr;
    AGB_CK(b->bufs.ensure("far", sizeof(FarArgs) * std::max<size_t>(1, b->far.size()), &v));
    b->d_far = (FarArgs *)v;
    AGB_CK(b->bufs.ensure("far_begin", sizeof(long long) * (b->far.size() + 1), &v));
    b->d_far_begin = (long long *)v;
    AGB_CK(b->bufs.ensure("near", sizeof(NearInst) * std::max<size_t>(1, b->near.size()), &v));
    b->d_near = (NearInst *)v;
    AGB_CK(b->bufs.ensure("near_begin", sizeof(long long) * b->near_begin.size(), &v));
    b->d_near_begin = (long long *)v;
    AGB_CK(b->bufs.ensure("counters", kCounters * sizeof(unsigned long long), &v));
    b->d_counters = (unsigned long long *)v;
    for (FarArgs &a : b->far) a.edge_counters = b->d_counters + 4;
    AGB_CK(b->bufs.ensure("reduce", sizeof(ReduceInst) * std::max<size_t>(1, b->red.size()), &v));
    b->d_red = (ReduceInst *)v;
    AGB_CK(b->bufs.ensure("reduce_begin", sizeof(long long) * b->red_begin.size(), &v));
    b->d_red_begin = (long long *)v;
    if (b->far.empty()) b->far_begin.assign(1, 0);
    ag_status st = batch_set_near_shape(b.get(), 0);
    if (st != AG_OK) return st;
    if (o.autotune) {
        st = batch_autotune(b.get());
        if (st != AG_OK) return st;
    } else {
        st = batch_upload_far(b.get(), false);
        if (st != AG_OK) return st;
        b->tune = ag_tuning{};
        b->tune.far_tile = 512;
        b->tune.near_shape = 0;
    }
    // final near unit table for the chosen shape
    st = batch_set_near_shape(b.get(), b->tune.near_shape);
    if (st != AG_OK) return st;
    // capture the run as a graph on a private stream
    cudaStream_t cs;
    AGB_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    AGB_CK(cudaStreamSynchronize(us));
    AGB_CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    st = batch_launch(b.get(), cs, b->tune.far_tile, b->tune.near_shape, nullptr, nullptr, nullptr, true);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (st != AG_OK) { if (g) cudaGraphDestroy(g); return st; }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    b->graph = g;
    AGB_CK(cudaGraphInstantiate(&b->exec, g, 0));
    *out = b.release();
    return AG_OK;
}

ag_status ag_batch_create(ag_context *ctx, const ag_problem *const *problems, int32_t n, const ag_opts *opts,
                          ag_batch **out)
{
    if (!ctx) return invalid("ag_batch_create: bad argument");
    return batch_create(ctx, problems, n, opts, ctx->stream, out);
}

ag_status ag_batch_run(ag_batch *b, void *stream)
{
    if (!b) return invalid("null batch");
    cudaStream_t s = stream ? (cudaStream_t)stream : b->ctx->stream;
    AGB_CK(cudaGraphLaunch(b->exec, s));
    return AG_OK;
}

const float *ag_batch_device_maps(const ag_batch *b, int32_t i)
{
    if (!b || i < 0 || i >= (int32_t)b->plans.size()) return nullptr;
    return b->plans[i]->maps32;
}

ag_status ag_batch_download(ag_batch *b, int32_t i, float *host_maps)
{
    if (!b || !host_maps || i < 0 || i >= (int32_t)b->plans.size()) return invalid("ag_batch_download: bad argument");
    const ag_plan *pl = b->plans[i].get();
    const size_t n_out = (size_t)pl->dp.n_maps + pl->floating + pl->constriction;
    AGB_CK(cudaMemcpyAsync(host_maps, pl->maps32, n_out * (size_t)pl->dp.P * sizeof(float), cudaMemcpyDefault,
                           b->ctx->stream));
    AGB_CK(cudaStreamSynchronize(b->ctx->stream));
    return AG_OK;
}

ag_status ag_batch_tuning(const ag_batch *b, ag_tuning *out)
{
    if (!b || !out) return invalid("null argument");
    *out = b->tune;
    return AG_OK;
}

ag_status ag_batch_destroy(ag_batch *b)
{
    if (!b) return AG_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
    return AG_OK;
}

ag_status ag_maps_compute_batch(ag_context *ctx, const ag_problem *const *problems, int32_t n, const ag_opts *opts,
                                float *const *maps)
{
    if (!maps) return invalid("null maps");
    if (!ctx || !problems || n < 1) return invalid("ag_maps_compute_batch: bad argument");
    for (int i = 0; i < n; i++)
        if (!problems[i] || !maps[i]) return invalid("ag_maps_compute_batch: null problem or output");
    const bool pipelined = n >= 8 && !(opts && opts->autotune);
    if (!pipelined) {
        ag_batch *b = nullptr;
        ag_status st = ag_batch_create(ctx, problems, n, opts, &b);
        if (st != AG_OK) return st;
        std::unique_ptr<ag_batch, ag_status (*)(ag_batch *)> guard(b, ag_batch_destroy);
        st = ag_batch_run(b, nullptr);
        for (int i = 0; st == AG_OK && i < n; i++) st = ag_batch_download(b, i, maps[i]);
        return st;
    }
    // Eight groups of instances, each a batch of its own: group g+1's plans are
    // built on the host (uploads on a stream of their own) while group g's
    // graph runs on the context's stream, and each group's maps are copied
    // back on the copy stream as soon as its graph is done.  Groups take the
    // instances round-robin by decreasing work, so they are of similar size.
    AGB_CK(cudaSetDevice(ctx->device));
    for (int i = 0; i < n; i++) {  // before any launch, with the caller's instance numbers
        const ag_status vs = validate(problems[i]);
        if (vs != AG_OK) {
            set_last_error("instance " + std::to_string(i) + ": " + ag_last_error());
            return vs;
        }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    auto work = [&](int i) {
        const ag_problem *p = problems[i];
        return (double)p->n1[0] * p->n1[1] * p->n1[2] * (double)(p->n_atoms + 64);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
    const int G = std::min(8, n);
    std::vector<std::vector<int>> groups(G);
    for (int k = 0; k < n; k++) groups[k % G].push_back(order[k]);
    cudaStream_t us = nullptr;
    AGB_CK(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking));
    std::vector<cudaEvent_t> done(G, nullptr);
    std::vector<ag_batch *> batches(G, nullptr);
    ag_status st = AG_OK;
    cudaError_t ce = cudaSuccess;
    for (int g = 0; g < G && st == AG_OK; g++) {
        std::vector<const ag_problem *> ps;
        for (int i : groups[g]) ps.push_back(problems[i]);
        st = batch_create(ctx, ps.data(), (int)ps.size(), opts, us, &batches[g]);
        if (st != AG_OK) break;
        st = ag_batch_run(batches[g], ctx->stream);
        if (st != AG_OK) break;
        if ((ce = cudaEventCreateWithFlags(&done[g], cudaEventDisableTiming)) != cudaSuccess ||
            (ce = cudaEventRecord(done[g], ctx->stream)) != cudaSuccess)
            break;
    }
    // copies after every launch: a copy into pageable memory blocks the host,
    // which must not hold up the building of later groups
    for (int g = 0; g < G && st == AG_OK && ce == cudaSuccess; g++) {
        if ((ce = cudaStreamWaitEvent(ctx->copy, done[g], 0)) != cudaSuccess) break;
        for (size_t k = 0; k < groups[g].size() && ce == cudaSuccess; k++) {
            const ag_plan *pl = batches[g]->plans[k].get();
            ce = cudaMemcpyAsync(maps[groups[g][k]], pl->maps32,
                                 ((size_t)pl->dp.n_maps + pl->floating + pl->constriction) * (size_t)pl->dp.P * sizeof(float),
                                 cudaMemcpyDefault, ctx->copy);
        }
    }
    const cudaError_t se = cudaStreamSynchronize(ctx->copy);
    for (ag_batch *b : batches) ag_batch_destroy(b);
    for (cudaEvent_t e : done)
        if (e) cudaEventDestroy(e);
    cudaStreamDestroy(us);
    if (st != AG_OK) return st;
    if (ce != cudaSuccess) return cuda_fail(ce, "ag_maps_compute_batch");
    if (se != cudaSuccess) return cuda_fail(se, "cudaStreamSynchronize");
    return AG_OK;
}

}  // extern "C"
