/*
 * autogrid_b200.h -- C ABI of the B200-native AutoGrid4 map engine.
 *
 * The reference (AutoGrid 4.2.8) has no library interface: its hot path is the
 * inline per-grid-point loop of main() (main.cpp:2785-3464), fed by globals
 * that the GPF/PDBQT/parameter front end fills (main.cpp:778-2736) and read by
 * the map writers (main.cpp:3481-3546).  This header is the seam a maintainer
 * would cut there:
 *
 *   front end  : ag_job_load()          <- main.cpp:214-2776 (GPF, parameter
 *                                          library, receptor, tables, bond vectors)
 *   hot path   : ag_maps_compute*()     <- main.cpp:2805-3464 (grid-point loop)
 *   back end   : ag_job_write_maps_*()  <- main.cpp:3481-3565 (map files, summary)
 *
 * Plain C types only; every pointer is host memory unless a function says
 * otherwise.  Errors are returned as ag_status codes (the reference calls
 * exit(1) through print_error(FATAL_ERROR), main.cpp:172-176); the message is
 * available from ag_last_error().  One host thread per context.
 */
#ifndef AUTOGRID_B200_H
#define AUTOGRID_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AG_ABI_VERSION 2   /* 2: ag_stats gained the far-field bin counters */

/* Table geometry of the reference build (-DUSE_8A_NBCUTOFF):
 * NEINT = NBC*A_DIV = 8*128 (constants.h:149-160), NDIEL = 64*128
 * (constants.h:170-171).  Bin of a distance r is (int)(r*A_DIV)
 * (autogrid.h:89). */
#define AG_A_DIV        128
#define AG_NEINT        1024
#define AG_NDIEL        8192
#define AG_NBC          8.0
#define AG_MAX_MAPS     128      /* autocomm.h:93-94 */
#define AG_MAX_REC_TYPES 20      /* autogrid.h:98 NUM_RECEPTOR_TYPES */
#define AG_MAX_ATOMS    100000   /* autogrid.h:58 AG_MAX_ATOMS */
#define AG_MAX_GRID_PTS 1025     /* autocomm.h:87 */

typedef enum ag_status {
    AG_OK               = 0,
    AG_ERR_INVALID      = 1,  /* inconsistent problem / bad argument            */
    AG_ERR_FATAL_INPUT  = 2,  /* a reference FATAL_ERROR condition (GPF, PDBQT,
                                 parameters); message in ag_last_error()        */
    AG_ERR_NO_CLOSEST_H = 3,  /* main.cpp:3011-3014 "no closestH atom was found" */
    AG_ERR_UNSUPPORTED  = 4,  /* requested a mode this build does not provide   */
    AG_ERR_CUDA         = 5,  /* CUDA runtime error; message names the call      */
    AG_ERR_NO_DEVICE    = 6,  /* no CUDA device / extension not usable          */
    AG_ERR_TOO_LARGE    = 7,  /* size beyond a stated limit                      */
    AG_ERR_IO           = 8,  /* file could not be opened or written            */
    AG_ERR_TIMEOUT      = 9   /* bounded wait on the device expired              */
} ag_status;

/* hbond classes, parameters.h:36-37 enum hbond_type */
enum { AG_HB_NON = 0, AG_HB_DS = 1, AG_HB_D1 = 2, AG_HB_AS = 3, AG_HB_A1 = 4,
       AG_HB_A2 = 5, AG_HB_AD = 6 };

/*
 * One receptor/box instance: a flat structure-of-arrays image of the globals
 * the reference's grid loop reads (main.cpp:360-379 atoms, :289-315 MapObject,
 * ad4_shared/structs.h:257-268 EnergyTables).  All arrays are owned by the
 * caller.  Coordinates are already centred on the grid centre, exactly as the
 * reference leaves coord[][] after the gridcenter keyword (main.cpp:1135-1139).
 */
typedef struct ag_problem {
    /* receptor atoms, in PDBQT file order */
    int32_t        n_atoms;
    const double  *coord;        /* [n_atoms*3]  x,y,z (Angstrom, centred)        */
    const double  *charge;       /* [n_atoms]                                      */
    const double  *vol;          /* [n_atoms]    atomic fragmental volume          */
    const double  *solpar;       /* [n_atoms]    atomic solvation parameter        */
    const int32_t *rec_type;     /* [n_atoms]    receptor type index               */
    const int32_t *hbond;        /* [n_atoms]    AG_HB_*                           */
    const int32_t *rexp;         /* [n_atoms]    D1 directionality exponent        */
    const double  *rvector;      /* [n_atoms*3]  bond vector (main.cpp:2301-2659)  */
    const double  *rvector2;     /* [n_atoms*3]  lone-pair plane normal (A2)       */
    const uint8_t *disorder;     /* [n_atoms]    disorder_h flags (main.cpp:2684)  */

    /* grid: n1 = npts+1 (odd) points per axis, icoord = i - ne, c = icoord*spacing */
    int32_t n1[3];
    int32_t ne[3];
    double  spacing;

    /* maps: indices 0..n_atom_maps-1 are ligand-type maps (with their
     * desolvation partner maps when separate_desolvation_maps is on); the
     * electrostatic and desolvation maps sit at elec_map / dsolv_map
     * (GPF order, main.cpp:1505-1544), -1 when not requested. */
    int32_t        n_rec_types;
    int32_t        n_atom_maps;
    int32_t        n_maps;
    int32_t        elec_map;
    int32_t        dsolv_map;
    const int32_t *map_is_covalent;  /* [n_atom_maps] */
    const int32_t *map_is_hbonder;   /* [n_atom_maps] */
    const int32_t *map_hbond;        /* [n_atom_maps] AG_HB_* of the probe type */
    const double  *map_solpar_probe; /* [n_atom_maps] */
    const double  *map_vol_probe;    /* [n_atom_maps] */

    /* lookup tables, as the reference stores them */
    const float   *e_vdw_hb;     /* [n_rec_types][n_atom_maps][AG_NEINT] float    */
    const double  *sol_fn;       /* [AG_NDIEL] coeff_desolv*exp(-r^2/(2*3.6^2))   */
    const double  *r_epsilon_fn; /* [AG_NDIEL] 332/eps(r) (dddiel only)            */

    /* scalars */
    int32_t dddiel;              /* distance-dependent dielectric (GPF dielectric <0) */
    double  invdielcal;          /* 332/diel for a constant dielectric            */
    double  coeff_estat;         /* AD4.coeff_estat                                */
    double  solpar_q;            /* qasp                                           */
    int32_t disorder_h;
    int32_t hydrogen_type;       /* receptor index of type "HD", -1 if absent      */
    int32_t separate_desolvation_maps;
    double  cov_pos[3];          /* covalent attachment point (centred)           */
    double  cov_half_width;
    double  cov_barrier;
    int32_t floating_grid;       /* fmap: distance to the nearest atom            */
    int32_t constriction_grid;   /* cmap: atoms within constriction_cutoff        */
    double  constriction_cutoff;
    /* 'map_receptor_interior off' (main.cpp:1642-1656), which the reference
     * supports in its USE_BHTREE build: a grid point with a receptor atom within
     * 1.5 A (BH_collision_dist, main.cpp:346) is a collision -- LOOP 1 is
     * skipped there, so its e-map value is 0 and its floating-grid value 1.5
     * (main.cpp:2907-2940) -- and the constriction grid counts the atoms within
     * the cutoff with the BH tree's single-precision test (bhtree.cpp:338-366,
     * main.cpp:2894-2899).  The test: float differences of the float grid point
     * and float atom coordinates, each within the cutoff, and their float
     * squared sum not above the float squared cutoff.  0 (default): the receptor
     * interior is mapped.  Drop-in path only (ag_maps_compute*, plans). */
    int32_t report_collisions;
} ag_problem;

enum { AG_PREC_FP32 = 0,   /* production path                                  */
       AG_PREC_FP64 = 1 }; /* FP64 GPU twin: the stated error oracle           */
enum { AG_TABLE_NEAREST = 0,   /* reference nearest-bin tables (drop-in)       */
       AG_TABLE_LINEAR = 1 }; /* linear interpolation between bins: the
                                 differentiable mode (ag_diff_*)               */

typedef struct ag_opts {
    int32_t precision;   /* AG_PREC_*                                          */
    int32_t table_mode;  /* AG_TABLE_*                                         */
    int32_t autotune;    /* batches: 1 = time tile/brick shapes at creation,   */
                         /* 0 = use the defaults                               */
    int32_t serial;      /* plans / one-shot calls: 1 = every kernel in       */
                         /* sequence on one stream (same work; for timing     */
                         /* kernels alone), 0 = far and near fields overlap   */
    int32_t reserved[4]; /* zero                                               */
} ag_opts;

/* Diagnostics of the last compute or plan run on a context (FP32 path);
 * ag_context_stats() waits for that run to finish. */
typedef struct ag_stats {
    int64_t near_pairs;        /* (point, atom) pairs inside 8 A evaluated       */
    int64_t fp64_fallbacks;    /* pairs re-evaluated in FP64 because an FP32
                                  distance fell within its error bound of a
                                  bin edge, the cutoff or an angular branch     */
    int64_t far_pairs;         /* e-map pairs evaluated by the far-field kernel  */
    int32_t gpu_launches;      /* kernels launched by the call                   */
    int32_t reserved;
    double  kernel_ms;         /* device time of the call's kernels (events)    */
    double  far_ms;            /* device time of the far-field e-map kernel      */
    double  text_ms;           /* device time of the last ag_maps_format's
                                  kernels (measure, scan and write passes)      */
    int64_t text_bytes;        /* bytes of map text that call produced          */
    double  table_ms;          /* device time of the last ag_tables_build        */
    /* Far-field table bins (e map, pairs beyond 8 A, distance-dependent
     * dielectric).  Every far pair's bin equals the reference's
     * (int)(r*A_DIV) of main.cpp:2951-2956: a pair whose FP32 distance lies
     * within its error bound of a bin edge is resolved in FP64. */
    int64_t far_edge_pairs;    /* far pairs resolved in FP64                     */
    int64_t far_fp32_bin_errors; /* of those, pairs whose plain FP32 bin
                                  floor(A_DIV*r) differed from the exact bin    */
    int64_t far_fp64_ties;     /* of those, pairs whose FP64 squared distance
                                  lay within 1e-12 of the edge; their bin is
                                  the reference expression's (nested hypot) in
                                  CUDA's libm, which may differ from the host
                                  libm's by one ulp of r                        */
    double  fixup_ms;          /* device time of the far-field fix-up kernel
                                  (part of far_ms; plans only)                  */
    double  near_ms;           /* device time from the first to the last
                                  near-field launch (ag_plan_run; with
                                  ag_opts.serial the near kernels' own time,
                                  otherwise overlapped with the far field)      */
} ag_stats;

typedef struct ag_context ag_context;

/* Library / device --------------------------------------------------------- */
const char *ag_last_error(void);
int32_t     ag_abi_version(void);
ag_status   ag_context_create(int32_t device, ag_context **out);
ag_status   ag_context_destroy(ag_context *ctx);
ag_status   ag_context_stats(const ag_context *ctx, ag_stats *out);
/* Device memory the context keeps for reuse: the 256 MiB blocks of destroyed
 * batches (ag_batch_destroy, and the groups of ag_maps_compute_batch), which
 * later batches take again instead of allocating.  The cache holds at most
 * what the largest batch call had in use at once; ag_context_trim frees it
 * (released may be null) and ag_context_destroy frees it too. */
ag_status   ag_context_cached_bytes(ag_context *ctx, int64_t *bytes);
ag_status   ag_context_trim(ag_context *ctx, int64_t *released);

/*
 * Hot path (replaces main.cpp:2805-3464).
 *
 * maps: [problem->n_maps][n1[2]][n1[1]][n1[0]] with X fastest, one contiguous
 * array per map, in the reference's gridmap order (main.cpp:321-322),
 * followed by the floating-grid map (Angstrom) and then the constriction map
 * (atom counts) when the problem asks for them (main.cpp:2947-2966).  The
 * problem arrays are host memory; `maps` may be host (pinned or pageable) or
 * device memory (CUDA unified addressing decides).  Device buffers are owned by
 * the context and reused across calls; the call returns when the maps are in
 * place.
 */
ag_status ag_maps_compute(ag_context *ctx, const ag_problem *problem,
                          const ag_opts *opts, float *maps);
/* Same, FP64 output (opts->precision must be AG_PREC_FP64). */
ag_status ag_maps_compute_f64(ag_context *ctx, const ag_problem *problem,
                              const ag_opts *opts, double *maps);

/*
 * One z-slab of the map set: grid planes [z0, z1) of every map (FP32), the
 * shard a device computes when a map set is split across GPUs.  The
 * reference parallelises its grid loop over the same axis (one OpenMP task
 * per z-plane, main.cpp:2805); a slab's points need every atom but nothing of
 * the other planes, so shards need no exchange.  z0 must be a multiple of 8
 * and z1 a multiple of 8 or n1[2] (AG_ERR_INVALID otherwise).  maps:
 * [n_out][z1-z0][n1[1]][n1[0]] (n_out as for ag_maps_compute), host or device
 * memory.  The planes equal those of ag_maps_compute bit for bit.  The
 * context's device is made current for the call and the caller's restored.
 */
ag_status ag_maps_compute_zslab(ag_context *ctx, const ag_problem *problem,
                                const ag_opts *opts, int32_t z0, int32_t z1, float *maps);

/*
 * Device-resident plan: the problem is validated and uploaded once, device
 * scratch (cell list, sorted atom tiles, padded tables) is allocated once,
 * and ag_plan_run() only launches kernels on `stream` (a cudaStream_t, or
 * NULL for the context's stream); results stay in plan-owned device memory.
 */
typedef struct ag_plan ag_plan;
ag_status    ag_plan_create(ag_context *ctx, const ag_problem *problem,
                            const ag_opts *opts, ag_plan **out);
ag_status    ag_plan_run(ag_plan *plan, void *stream);
/* ag_plan_run for grid planes [z0, z1) only (bounds as ag_maps_compute_zslab);
 * the planes land at their places in the plan's device maps. */
ag_status    ag_plan_run_zslab(ag_plan *plan, int32_t z0, int32_t z1, void *stream);
const float *ag_plan_device_maps(const ag_plan *plan);   /* device pointer  */
size_t       ag_plan_points(const ag_plan *plan);        /* n1x*n1y*n1z     */
ag_status    ag_plan_download(ag_plan *plan, float *host_maps);
ag_status    ag_plan_destroy(ag_plan *plan);

/*
 * Energy tables on the device: the table fill of main.cpp:2040-2276 (LJ 12-6 /
 * H-bond 12-10 pair tables with the EINTCLAMP clamp and the +-smooth/2 bin
 * minimum filter, the desolvation table) and the Mehler-Solmajer dielectric
 * of main.cpp:1607-1639, from the per-(map, receptor type) parameters the
 * parameter library and the nbp_r_eps / nbp_coeffs keywords produce
 * (ag_job_table_params).  Outputs as ag_problem stores the tables:
 * e_vdw_hb [n_rec_types][n_atom_maps][AG_NEINT], sol_fn and r_epsilon_fn
 * [AG_NDIEL] (r_epsilon_fn may be NULL with a constant dielectric); host or
 * device memory.  FP64 arithmetic in the reference's order, CUDA pow/exp.
 * A problem whose three table pointers are device memory is accepted by
 * ag_maps_compute*, ag_plan_create and ag_batch_create (packed on the device)
 * and by ag_diff_create* (read once at creation).  AG_ERR_FATAL_INPUT on a NaN
 * coefficient or a zero exponent (main.cpp:2166-2183).
 */
typedef struct ag_table_params {
    int32_t        n_rec_types;
    int32_t        n_atom_maps;
    const double  *cA, *cB;          /* [n_atom_maps][n_rec_types]; both 0: from Rij, epsij */
    const double  *Rij, *epsij;      /* [n_atom_maps][n_rec_types]                          */
    const int32_t *xA, *xB;          /* [n_atom_maps][n_rec_types] exponents                */
    const int32_t *map_is_covalent;  /* [n_atom_maps]: table left zero                     */
    double         r_smooth;         /* GPF smooth (Angstrom)                               */
    double         coeff_desolv;     /* AD4.coeff_desolv                                    */
    int32_t        dddiel;           /* 1: distance-dependent dielectric                    */
} ag_table_params;
ag_status ag_tables_build(ag_context *ctx, const ag_table_params *params, float *e_vdw_hb, double *sol_fn,
                          double *r_epsilon_fn);

/*
 * Map-file bodies formatted on the device (replaces the text loop of
 * main.cpp:3481-3519), byte for byte what the reference's fprintf writes:
 *   energy maps     "0\n" when fabs(e) < 1e-4 (PRECISION, autogrid.h:68),
 *                   else "%.3f\n" of (float)round3dp(e) (main.cpp:84-86);
 *   floating grid   "%.3f\n" of (float)round3dp(r_min);
 *   constriction    "%d\n" of the atom count.
 * `device_maps` holds the n_out = problem->n_maps (+1 floating, +1
 * constriction) output maps of ag_maps_compute's layout in DEVICE memory,
 * FP32 (elem_size 4) or FP64 (8); for example ag_plan_device_maps().  On
 * return *text points to the bodies, map after map, in pinned host memory
 * owned by the context (valid until its next text call or
 * ag_context_destroy); map_bytes[k] (n_out entries) is the length of map k's
 * body; emin/emax (n_maps entries each, may be NULL) receive each energy
 * map's extrema over the unrounded values (main.cpp:3494-3495).
 */
ag_status ag_maps_format(ag_context *ctx, const ag_problem *problem, const void *device_maps,
                         int32_t elem_size, const char **text, size_t *map_bytes, double *emin,
                         double *emax);
/* ag_maps_compute (FP32) or ag_maps_compute_f64 (opts->precision FP64) and
 * ag_maps_format in one call, the maps never leaving the device. */
ag_status ag_maps_compute_text(ag_context *ctx, const ag_problem *problem, const ag_opts *opts,
                               const char **text, size_t *map_bytes, double *emin, double *emax);

/*
 * Electrostatic map for callers that cannot allocate device memory.  No
 * counterpart in the reference (which has no library interface).  Meant for
 * processes whose device memory is owned by their own pool allocator, or
 * serving loops that may not call cudaMalloc/cudaFree (cudaFree synchronises
 * the device) between requests.  Computes the e map of LOOP 1
 * (main.cpp:2940-2982) from caller-owned DEVICE buffers -- d_coord
 * [n_atoms*3] centred coordinates, d_charge [n_atoms], d_r_epsilon_fn
 * [AG_NDIEL] (dddiel only) -- into the caller-owned device map d_emap
 * [n1z*n1y*n1x] floats, on `stream` (a cudaStream_t; NULL = legacy default
 * stream), and returns once the work is enqueued.
 *
 * Scratch lives in one static device array of AG_NOALLOC_SCRATCH_BYTES that
 * every GPU which loads this entry point's module keeps until process exit;
 * grids that do not fit (about 7.5 million points at 10,000 atoms) are
 * rejected with AG_ERR_TOO_LARGE.  The first call on a device resolves the
 * array's device address (cudaGetSymbolAddress) and keeps it for the process,
 * so make that first call before any stream capture, and do not use this entry
 * point on a device after a cudaDeviceReset of it.  All calls share the array:
 * calls that overlap on the GPU (other streams, other host threads) race.
 * Every scratch word read is written earlier in the same call, so nothing
 * needs clearing.  `stream` must belong to `device` (AG_ERR_INVALID
 * otherwise); the caller's current device is restored on return.  Table bins
 * follow the far-field bin guard of ag_maps_compute (no statistics).
 */
#define AG_NOALLOC_SCRATCH_BYTES (32u << 20)
ag_status ag_emap_compute_noalloc(int32_t device, int32_t n_atoms, const double *d_coord,
                                  const double *d_charge, const int32_t n1[3], double spacing,
                                  int32_t dddiel, const double *d_r_epsilon_fn, double invdielcal,
                                  double coeff_estat, float *d_emap, void *stream);

/*
 * Batched ensemble: many independent receptor/box instances (uneven atom
 * counts and grids) computed by one persistent launch per kernel kind, each
 * CTA taking (instance, tile) work units from an atomic counter.  The kernel
 * sequence is captured once in a CUDA graph.  With opts->autotune set,
 * ag_batch_create() also runs the autotuner: it times the far-field atom-tile
 * size and chunking and the near-field brick shape on this batch and keeps
 * the fastest.  No counterpart
 * in the reference, which computes one box per process.  FP32 path only.
 * Instances that ask for the floating or constriction grid get them after
 * their energy maps, as ag_maps_compute lays them out; they depend on the
 * geometry only and are computed once, at creation.
 */
typedef struct ag_batch ag_batch;
typedef struct ag_tuning {
    int32_t far_tile;         /* atoms per shared-memory tile (256, 512, 1024)     */
    int32_t far_chunked;      /* 1: atoms split in 2048-atom chunks per unit       */
    int32_t near_shape;       /* 0: 8x8x4, 1: 8x4x8, 2: 4x8x8 points per brick     */
    int32_t candidates;       /* configurations timed                             */
    double  far_ms, near_ms;  /* device time of the chosen far / near launches    */
    double  far_ms_default, near_ms_default;  /* same with the untuned defaults   */
} ag_tuning;
ag_status    ag_batch_create(ag_context *ctx, const ag_problem *const *problems, int32_t n,
                             const ag_opts *opts, ag_batch **out);
ag_status    ag_batch_run(ag_batch *batch, void *stream);
const float *ag_batch_device_maps(const ag_batch *batch, int32_t i);
ag_status    ag_batch_download(ag_batch *batch, int32_t i, float *host_maps);
ag_status    ag_batch_tuning(const ag_batch *batch, ag_tuning *out);
/* Destroy a batch before its context.  Its device memory goes back to the
 * context, which reuses it for later batches and frees it in
 * ag_context_destroy. */
ag_status    ag_batch_destroy(ag_batch *batch);
/* One-shot: create, run, download every instance's maps (maps[i] host or
 * device, [n_out_i][P_i] each: the energy maps, then fmap/cmap when asked
 * for), destroy.  From 8 instances on (without
 * autotuning) the instances run as 8 groups, each its own batch: a group's
 * plans are built on the host while the previous group computes, and each
 * group's maps are copied back while later groups compute.  Results are those
 * of one batch without autotuning. */
ag_status    ag_maps_compute_batch(ag_context *ctx, const ag_problem *const *problems, int32_t n,
                                   const ag_opts *opts, float *const *maps);

/*
 * Differentiable mode.  No counterpart in the reference (which has no
 * gradients).  The maps of the hot path with every distance table read by
 * linear interpolation between bins, the short-range terms switched to zero
 * over the last bin before the 8 A cutoff, the D1 ramp evaluated for every D1
 * pair and the two A2 angular branches made to meet at cos_theta = 0, so the
 * maps are continuous in the receptor coordinates and charges.  Discrete
 * choices are frozen: each point's closest DS/D1 atom (kept from an earlier
 * forward on request), the bonded neighbours behind the bond vectors (see
 * ag_job_bond_vectors) and, for the adjoint, the atoms attaining each H-bond
 * min/max.  The nearest-bin drop-in (ag_maps_compute) is unchanged.
 *
 * Limits: at most 16 maps besides the e map, at most 8 of which keep an H-bond
 * min/max (AG_ERR_UNSUPPORTED otherwise).
 *
 * Arrays: coord [3N] centred (the problem's frame), charge [N], rvector and
 * rvector2 [3N], all FP64 host memory.  Maps and map gradients are
 * [n_maps][P] in the precision of opts->precision (float or double); P =
 * n1x*n1y*n1z.
 *
 * Conformers: an object may hold K coordinate sets (conformers) of the same
 * receptor -- same atoms, types, tables and grid -- evaluated together, each
 * forward and each backward one launch per kernel over all K.  Per-conformer
 * arrays are then stacked: maps [K][n_maps][P], closest H [K][P], gradients
 * [K][3N] / [K][N].
 */
typedef struct ag_diff ag_diff;
/* Bind a problem (copied: atoms, types, tables); opts->precision selects the
 * FP32 kernels or their FP64 twin, opts->table_mode must be AG_TABLE_LINEAR. */
ag_status   ag_diff_create(ag_context *ctx, const ag_problem *problem, const ag_opts *opts,
                           ag_diff **out);
/* Same with n_conformers (1..4096) conformers, each starting at the
 * problem's coordinates. */
ag_status   ag_diff_create_batch(ag_context *ctx, const ag_problem *problem, const ag_opts *opts,
                                 int32_t n_conformers, ag_diff **out);
int32_t     ag_diff_conformers(const ag_diff *d);
/* Replace atom coordinates, charges and bond vectors of conformer 0 / of
 * conformer k (NULL keeps the current). */
ag_status   ag_diff_set_atoms(ag_diff *d, const double *coord, const double *charge,
                              const double *rvector, const double *rvector2);
ag_status   ag_diff_set_conformer(ag_diff *d, int32_t k, const double *coord, const double *charge,
                                  const double *rvector, const double *rvector2);
/* Compute all maps.  keep_closest_h = 1 reuses the closest DS/D1 atoms of the
 * previous forward (0, or no previous forward: search them at the current
 * coordinates, as main.cpp:2986-3015 does).  device_out: a device buffer of
 * [n_maps][P] elements to write, or NULL for the object's own buffer.
 * Returns when the maps are in place. */
ag_status   ag_diff_forward(ag_diff *d, int32_t keep_closest_h, void *device_out);
const void *ag_diff_device_maps(const ag_diff *d);            /* own buffer     */
ag_status   ag_diff_download(ag_diff *d, void *host_maps);     /* own buffer     */
/* [P] file index of each point's closest DS/D1 atom (-1: none needed). */
ag_status   ag_diff_closest_h(ag_diff *d, int32_t *host_out);
/* Adjoint of the last forward for L with dL/d(maps) = grad_maps ([n_maps][P],
 * device memory if grad_on_device, else host).  Writes dL/d(coord) through the
 * pair terms only, dL/d(charge), dL/d(rvector), dL/d(rvector2) (FP64 host
 * arrays, any may be NULL).  The bond vectors' own dependence on the
 * coordinates is ag_job_bond_vectors_backward.  Pair terms are recomputed, not
 * stored. */
ag_status   ag_diff_backward(ag_diff *d, const void *grad_maps, int32_t grad_on_device,
                             double *g_coord, double *g_charge, double *g_rvector,
                             double *g_rvector2);
/* Device-resident atom updates.  ag_diff_set_bonds attaches a bond topology
 * (ag_job_bond_topology, host memory); ag_diff_set_atoms_device then takes
 * DEVICE arrays for every conformer at once -- coord [K][3N], charge [K][N]
 * (NULL keeps the charges) -- and rebuilds on the device the bond vectors (when
 * a topology is attached; otherwise they are kept) and the cell lists.  The
 * arrays must be ready when the call is made and may be reused once it
 * returns.  ag_diff_backward_device is ag_diff_backward with the map gradient
 * and the outputs in device memory: g_coord [K][3N] includes the bond vectors'
 * dependence on the coordinates when a topology is attached (the pair terms
 * only otherwise), g_charge [K][N]; either may be NULL. */
ag_status   ag_diff_set_bonds(ag_diff *d, const int32_t *topo);
ag_status   ag_diff_set_atoms_device(ag_diff *d, const double *coord, const double *charge);
ag_status   ag_diff_backward_device(ag_diff *d, const void *grad_maps, double *g_coord, double *g_charge);
/* Device times (ms) of the last forward (e map + short-range maps), of the
 * last closest-H search and of the last backward. */
ag_status   ag_diff_timing(const ag_diff *d, float *forward_ms, float *closest_h_ms,
                           float *backward_ms);
ag_status   ag_diff_destroy(ag_diff *d);

/* Front / back end (replaces main.cpp:214-2776 and :3481-3565) ------------- */
typedef struct ag_job ag_job;

/* Parse a GPF exactly as autogrid4 -p gpf -l glg would (relative file names
 * resolve against the current directory), read the receptor and parameter
 * library, build energy tables and bond vectors, open the map files and
 * write the .fld/.xyz files.  glg_path may be NULL (log to stdout). */
ag_status          ag_job_load(const char *gpf_path, const char *glg_path, ag_job **out);
const ag_problem  *ag_job_problem(const ag_job *job);
/* Write the map files (main.cpp:3481-3519) and the GLG extrema summary and
 * completion line (main.cpp:3530-3565) from FP32 or FP64 maps. */
ag_status          ag_job_write_maps_f32(ag_job *job, const float *maps);
ag_status          ag_job_write_maps_f64(ag_job *job, const double *maps);
/* Same files and GLG summary from bodies already formatted by
 * ag_maps_format / ag_maps_compute_text (map_bytes: one entry per output map;
 * emin/emax: one per energy map). */
ag_status          ag_job_write_text(ag_job *job, const char *text, const size_t *map_bytes,
                                     const double *emin, const double *emax);
/* Record a fatal error in the job's GLG ("Unsuccessful Completion"). */
void               ag_job_fail(ag_job *job, const char *message);
void               ag_job_free(ag_job *job);
/* Bond topology behind the bond vectors (frozen at load, main.cpp:2297-2659):
 * topo [n_atoms][7] = kind (AG_BOND_*), i1, i2, nb, nbr[3] per atom, the
 * atoms whose coordinates define rvector/rvector2 of that atom:
 *   AG_BOND_D1      rvector = unit(x - x[i1])                    (donor H)
 *   AG_BOND_A2_ONE  rvector = unit(x - x[i1]); with i2 >= 0,
 *                   rvector2 = unit(rvector x unit(x[i1] - x[i2]))
 *   AG_BOND_A2_DIS  rvector = unit(x - x[i1])
 *   AG_BOND_A2_TWO  rvector2 = unit(x[i2] - x[i1]), rvector = unit of the
 *                   component of x - x[i1] normal to rvector2
 *   AG_BOND_A1      rvector = -unit(mean over nbr[0..nb) of x - x[nbr])
 * For ag_diff_set_bonds. */
enum { AG_BOND_NONE = 0, AG_BOND_D1 = 1, AG_BOND_A2_ONE = 2, AG_BOND_A2_DIS = 3, AG_BOND_A2_TWO = 4,
       AG_BOND_A1 = 5 };
ag_status          ag_job_bond_topology(const ag_job *job, int32_t *topo);
/* The job's table parameters for ag_tables_build (arrays owned by the job). */
ag_status          ag_job_table_params(const ag_job *job, ag_table_params *out);
/* The job with Vina-potential tables in place of the AD4 ones: the table
 * fill of main.cpp:2081-2126 (compiled out of the reference build,
 * use_vina_potential = FALSE at main.cpp:263) with the xs radii of
 * read_parameter_library.cc:323-339 (1.8 A for other types), restated as
 * written.  The problem has the job's atoms, grid and atom maps only (the
 * reference drops the e and d maps and desolvation under Vina), no H-bond
 * directionality (plain sums) and no desolvation; it is owned by the job.
 * AG_ERR_UNSUPPORTED with separate_desolvation_maps. */
ag_status          ag_job_vina_problem(ag_job *job, const ag_problem **out);
/* Bond vectors (rvector, rvector2; [3N] each) at other coordinates coord
 * ([3N], the problem's centred frame; NULL = the job's own), keeping the
 * bonded neighbours the GPF load found (main.cpp:2320-2656: the same vector
 * arithmetic, the neighbour search frozen).  At the job's own coordinates the
 * result equals the problem's rvector/rvector2 bit for bit. */
ag_status          ag_job_bond_vectors(const ag_job *job, const double *coord, double *rvector,
                                       double *rvector2);
/* Adjoint of ag_job_bond_vectors at coord, in FP64:
 * g_coord += d(rvector, rvector2)/d(coord)^T (g_rvector, g_rvector2).
 * No reference counterpart (the reference has no gradients). */
ag_status          ag_job_bond_vectors_backward(const ag_job *job, const double *coord,
                                                const double *g_rvector, const double *g_rvector2,
                                                double *g_coord);

#ifdef __cplusplus
}
#endif
#endif /* AUTOGRID_B200_H */
