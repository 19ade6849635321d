/*
 * cipher_b200.h - C ABI of the B200 implementation of CIPHER's time-stepper
 * right-hand side.
 *
 * Plain pointers and sizes only.  Device pointers are CUDA global-memory
 * addresses on the context's device; `stream` is a cudaStream_t passed as
 * void* (NULL = legacy default stream).  Every entry point returns 0 on
 * success or one of the CIPHER_E_* codes; cipher_last_error() gives a
 * message for the calling thread.
 *
 * The two hot entry points replace the reference's PETSc callbacks:
 *   cipher_rhs      <- RHSFunction(TS, PetscReal, Vec X, Vec F, void *ctx)
 *                      src/cipher.c:20,27-681, registered at src/cipher.c:1107
 *   cipher_poststep <- PostStep(TS), active-set part src/cipher.c:869-974,
 *                      registered at src/cipher.c:1108
 */
#ifndef CIPHER_B200_H
#define CIPHER_B200_H

#include <stdint.h>
#include <stddef.h>
#include "cipher_problem.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* error codes                                                         */
/* ------------------------------------------------------------------ */
#define CIPHER_OK             0
#define CIPHER_E_ARG          1   /* invalid argument */
#define CIPHER_E_NOMEM        2   /* host or device allocation failed */
#define CIPHER_E_CAP          3   /* active-set superset above the cap; the
                                     reference asserts (src/cipher.c:968) */
#define CIPHER_E_NONFINITE    4   /* NaN/Inf in a state or error norm */
#define CIPHER_E_CUDA         5   /* CUDA runtime error */
#define CIPHER_E_TIMEOUT      6   /* a bounded device wait ran out */
#define CIPHER_E_UNSUPPORTED  7   /* configuration not implemented on device */
#define CIPHER_E_STEP         8   /* time step fell below the minimum */

const char *cipher_strerror(int code);
const char *cipher_last_error(void);

/* Contexts, steppers, batches and served requests take their device
 * buffers from a stream-ordered pool per device that keeps freed blocks for
 * reuse; this hands the pooled blocks of `device` back to the driver. */
int cipher_pool_trim(int device);

/* sizeof of the public structs, for binding generators to check their
 * mirrors: out[0..11] = tseries, rk, mobility, source, material, interface,
 * bc, problem, mesh, nucleus, output_field, config; returns how many were
 * written (at most n) */
int cipher_abi_sizes(int64_t *out, int n);

/* ------------------------------------------------------------------ */
/* host: problem description, meshes, initial state                    */
/* (the reference builds these in SetUpConfig/main/SetUpProblem,        */
/*  src/init.c:104-1716, src/cipher.c:1148-1231, src/init.c:1721-1830)  */
/* ------------------------------------------------------------------ */

/* allocate a problem with default parameters (src/init.c:1260-1327 defaults) */
cipher_problem *cipher_problem_new(int dim, int npf, int ncp, int nmat, int nf);
void cipher_problem_free(cipher_problem *p);
/* derive nsites, stoichiometry, maxsites after the tables are filled */
int cipher_problem_finalize(cipher_problem *p);
/* P = min(max_phase_neighbours, npf)  (src/init.c:1326-1343) */
int cipher_problem_set_cap(cipher_problem *p, int max_phase_neighbours);
cipher_aos_layout cipher_problem_aos_layout(const cipher_problem *p);

/* seeded grain-growth problem: periodic box of res[] cells, ngrains Voronoi
 * grains (splitmix64 seed), one material with chemicalenergy none, one
 * interface of the given energy, mobility and width */
int cipher_problem_grain_growth(int dim, const int32_t *res, int ngrains, int cap, uint64_t seed,
                                double energy, double mobility, double width,
                                double molarvolume, double temperature0,
                                cipher_problem **out);
/* feature bits of cipher_problem_grain_growth_multi */
#define CIPHER_GG_ACTIVATION  0x01u  /* T-dependent energy and mobility on every other interface */
#define CIPHER_GG_WIDTHS      0x02u  /* interface widths uniform in [3, 5] cells instead of 4 */

/* grain growth with several interfaces: the problem of
 * cipher_problem_grain_growth (energy 1, mobility 1, width 4, Vm 1e-5,
 * T0 500) with `ninterfaces` seeded interfaces (energy and mobility
 * prefactors uniform in [0.5, 1.5], plus the CIPHER_GG_* features), and every
 * grain pair a<b assigned a seeded interface in the upper triangle of
 * interfacelist, as the reference's parser fills it (src/init.c:1501).
 * Misorientation-dependent boundaries in the reference are such tables. */
int cipher_problem_grain_growth_multi(int dim, const int32_t *res, int ngrains, int cap, uint64_t seed,
                                      int ninterfaces, unsigned features, cipher_problem **out);

/* feature bits of cipher_problem_alloy */
#define CIPHER_ALLOY_SEGREGATION   0x01u  /* segregation potentials on grain and phase boundaries */
#define CIPHER_ALLOY_ITF_MOBILITY  0x02u  /* interface factors on the solute mobilities */
#define CIPHER_ALLOY_ACTIVATION    0x04u  /* T-dependent interface energy and mobility */
#define CIPHER_ALLOY_THERMAL       0x08u  /* specific heat, latent heat, conductivity */
#define CIPHER_ALLOY_SOURCES       0x10u  /* solute sinks in the precipitates and on grain boundaries */
#define CIPHER_ALLOY_WALLS         0x20u  /* x not periodic; chemical and thermal BCs on both walls */
#define CIPHER_ALLOY_TEMP_RATE     0x40u  /* imposed cooling rate */
#define CIPHER_ALLOY_MIXED_MODELS  0x80u  /* matrix calphaddis, precipitates calphad2sl */

/* seeded alloy problem: two matrix grains (Voronoi) with nprecip spherical
 * precipitates, ncp components, free-energy model `model` (quadratic,
 * calphaddis or calphad2sl: matrix 1:1, precipitates 2:1 sublattices) with
 * random coefficients, T = 700 K, interface width 4 cells, plus the
 * CIPHER_ALLOY_* features.  No counterpart in the reference (which reads
 * its tables from YAML); it fills the same tables. */
int cipher_problem_alloy(int dim, const int32_t *res, int model, int ncp, int nprecip, int cap, uint64_t seed,
                         unsigned features, cipher_problem **out);

/* nearest-centre Voronoi map under the periodic metric, x fastest; the
 * seeded centres are returned in centres[ngrains*3] when it is not NULL */
int cipher_voronoi(int dim, const int32_t *res, int ngrains, uint64_t seed, int32_t *voxel, double *centres);
double cipher_rand_uniform(uint64_t *state);

/* uniform leaf mesh; owned planes [slab_lo, slab_hi) of the slowest axis
 * plus a one-cell halo (pass 0, res[dim-1] for the whole domain) */
int cipher_mesh_uniform(const cipher_problem *p, int slab_lo, int slab_hi, cipher_mesh **out);
/* the whole-domain grid without face lists (O(1) memory): enough for a
 * device context, not for the host builders or the oracle */
int cipher_mesh_grid(const cipher_problem *p, cipher_mesh **out);
void cipher_mesh_free(cipher_mesh *m);

/* ------------------------------------------------------------------ */
/* adaptive meshes: a quadtree / octree forest over a brick of blocks  */
/* (the reference's p4est forest, src/cipher.c:1149-1159; its adaptation */
/*  src/cipher.c:1365-1586 and 1607-1829)                              */
/* ------------------------------------------------------------------ */

typedef struct cipher_forest cipher_forest;

/* nblocks[d] blocks per direction; leaves between levels lmin and lmax (a
 * level-l leaf spans 2^(lmax-l) finest cells, so the finest grid, which is
 * the grid of voxel maps and of cell_global, has nblocks[d]*2^lmax cells);
 * uniform at level linit to start with.  size = physical extent (NULL: one
 * unit per finest cell). */
int cipher_forest_create(int dim, const int32_t *nblocks, int lmin, int lmax, int linit, const int32_t *periodic,
                         const double *size, cipher_forest **out);
void cipher_forest_destroy(cipher_forest *f);
int64_t cipher_forest_nleaves(const cipher_forest *f);
/* per leaf: level and lower corner on the finest grid (corner[3*i+d]); either may be NULL */
int cipher_forest_leaves(const cipher_forest *f, int32_t *level, int32_t *corner);
int cipher_forest_resolution(const cipher_forest *f, int32_t *res);
/* the reference's marks (src/cipher.c:1380-1386): +1 (refine) where a leaf's
 * active set holds more than one phase, -1 (coarsen) elsewhere; X is the
 * reference AoS state of the leaves */
int cipher_forest_mark_active(const cipher_forest *f, const double *X, int ndof, int8_t *mark);
/* adapt by marks (+1 refine once, -1 coarsen a whole family of siblings, 0
 * keep) within [lmin, lmax], then 2:1 face balance; with Xold (AoS, ndof
 * doubles per leaf) a family whose first as_size dofs (the active set)
 * differ is kept.  The transfer plan is kept for the two calls below. */
int cipher_forest_adapt(cipher_forest *f, const int8_t *mark, const double *Xold, int ndof, int as_size);
/* new leaf i takes the mean of old leaves [src0[i], src0[i] + nsrc[i]) */
int cipher_forest_transfer_plan(const cipher_forest *f, int64_t *src0, int32_t *nsrc);
/* the finite-volume transfer of an AoS state (DMForestTransferVec): children
 * copy their parent, a coarsened family's mean goes to the parent */
int cipher_forest_transfer_aos(const cipher_forest *f, const double *Xold, int ndof, double *Xnew);
/* the mesh of the leaves: cells in leaf order with cellgeom = vol^(1/dim),
 * every interior face once (conforming faces, and the hanging faces between
 * a coarse leaf and each finer neighbour), boundary faces of non-periodic
 * sides labelled 2d+1 (low) / 2d+2 (high) */
int cipher_forest_mesh(const cipher_forest *f, cipher_mesh **out);

/* SetUpProblem active sets / phi / T in the reference AoS layout (host) */
int cipher_initial_state_aos(const cipher_problem *p, const cipher_mesh *m, double *X);

/* a diffuse-interface state of a Voronoi problem (host): every grain j whose
 * bisector with the cell's nearest grain i is closer than width/2 gets
 * weight f/(1-f), f = (1 - sin(pi d/width))/2, the owner weight 1, phi the
 * normalised weights; active sets are then united with the face neighbours'
 * as the per-step update does.  Returns CIPHER_E_CAP if a set exceeds P. */
int cipher_initial_state_diffuse_aos(const cipher_problem *p, const cipher_mesh *m, double width, double *X);

/* ------------------------------------------------------------------ */
/* device context                                                      */
/* ------------------------------------------------------------------ */

typedef struct cipher_ctx cipher_ctx;

enum { CIPHER_PREC_FP64 = 0,    /* plain FP64 drop-in */
       CIPHER_PREC_MIXED = 1 }; /* FP32 phi/T storage and stencil, FP64 chemistry */

/*
 * Device state layout (structure of arrays, plane-major, one plane per slot):
 *   AS  uint16 [P+1][stride]   plane 0 = active count n, planes 1..P = sorted ids
 *   MAP uint32 [P][stride]     face maps (uniform grids): for each active slot k
 *                              < n, bits 4q..4q+3 of word [k][cell] hold the
 *                              slot of the same phase in the neighbour across
 *                              face q (q = 2d: lower, 2d+1: upper neighbour
 *                              along d), or 15 where the neighbour lacks it or
 *                              the reference's face gate is off; words of
 *                              slots >= n are unspecified.  Derived from AS:
 *                              rebuilt by cipher_poststep,
 *                              cipher_state_from_aos and cipher_state_refresh.
 *                              Adapted meshes have none (map_planes 0).
 *   PF  real   [P][stride]     phase fractions of the active phases
 *   DP  double [D][stride]     diffusion potentials mu
 *   EX  double [P*S][stride]   explicit site potentials, slot g*S+s*D+c
 *   TM  real   [stride]        temperature
 * real = double (FP64) or float (MIXED).  Offsets are bytes from the state
 * base pointer; every plane starts on a 256-byte boundary.  The RHS vector F
 * uses the same layout; its AS and MAP regions are not written (the
 * reference's F is identically zero there).  AS and MAP together occupy
 * [as_offset, pf_offset): copying that range copies a state's sets.
 */
typedef struct cipher_state_layout {
    int64_t ncells;      /* owned cells */
    int64_t stride;      /* elements per plane (ncells rounded up) */
    int32_t pf_size, dp_size, ex_size, precision;
    int64_t as_offset, pf_offset, dp_offset, ex_offset, tm_offset;
    int64_t bytes;       /* total bytes of one state vector */
    int64_t map_offset;  /* MAP region (between AS and PF) */
    int32_t map_planes;  /* P (uniform grids) or 0 (adapted meshes) */
} cipher_state_layout;

/* create a context on `device` for problem p over mesh m (owned cells only;
 * ghosts are not used on one GPU) */
int cipher_ctx_create(const cipher_problem *p, const cipher_mesh *m, int precision, int device,
                      cipher_ctx **out);
void cipher_ctx_destroy(cipher_ctx *c);
int cipher_ctx_layout(const cipher_ctx *c, cipher_state_layout *out);

/* F = RHS(t, X) over all owned cells; X and F are device state vectors */
int cipher_rhs(cipher_ctx *c, double t, const void *X, void *F, void *stream);

/* which kernel an FP64 grain-growth context with a single interface uses:
 * the reference's operation order (default; bit-identical to the
 * reference), or the O(n) closed form of the pair and triple sums that the
 * mixed path uses, in FP64 (equal to the reference within rounding) */
enum { CIPHER_RHS_REFERENCE_ORDER = 0, CIPHER_RHS_CLOSED_FORM = 1 };
int cipher_ctx_set_rhs_form(cipher_ctx *c, int form);

/* per-step active-set update of X in place: Gibbs-simplex projection, prune
 * phi <= TOL, union with the face neighbours' pruned sets, reorder PF/EX.
 * Synchronises `stream`; returns CIPHER_E_CAP if a superset exceeds P. */
int cipher_poststep(cipher_ctx *c, void *X, void *stream);

/* synchronise `stream`, then read and clear the error flags the kernels
 * raise instead of trapping (bad active counts, cap overflow) */
int cipher_ctx_check(cipher_ctx *c, void *stream);

/* the SetUpProblem state (src/init.c:1721-1830) built on the device from
 * the voxel map (host, x fastest, one phase per cell): sets = own phase and
 * the face neighbours' phases, phi = 1 for the own phase, T = its
 * material's temperature0, then the face maps and the chemistry of
 * cipher_chem_init.  Returns CIPHER_E_CAP when a set exceeds P. */
int cipher_state_init_sharp(cipher_ctx *c, const int32_t *voxelphase, void *X, void *stream);

/* after a forest adaptation: Xdst (context dst, the new mesh) from Xsrc
 * (context src, the old mesh) by the forest's transfer plan (host arrays,
 * cipher_forest_transfer_plan): children copy their parent, a coarsened
 * family's mean goes to the parent (DMForestTransferVec,
 * src/cipher.c:1433).  Equal to cipher_forest_transfer_aos in FP64.
 * Synchronises `stream`. */
int cipher_state_transfer(cipher_ctx *dst, void *Xdst, const cipher_ctx *src, const void *Xsrc,
                          const int64_t *src0, const int32_t *nsrc, void *stream);

/* rebuild the face maps of X from its active sets, for callers that write
 * the AS planes themselves (the library's own producers keep them current) */
int cipher_state_refresh(cipher_ctx *c, void *X, void *stream);

/* chemistry of an initial state whose sets, phi and T are filled (device):
 * EX of every listed phase = SitepotentialExplicit(c0, T), mu = the summed
 * Sitepotential(c0, T) of the phase with the largest phi (the voxel's own
 * phase in a sharp state), as SetUpProblem does (src/init.c:1790-1823).
 * No-op without chemistry. */
int cipher_chem_init(cipher_ctx *c, void *X, void *stream);

/* grid and state description for the allocation-free entry point */
typedef struct cipher_grid_desc {
    int32_t dim;
    int32_t res[3];
    int32_t periodic[3];
    int32_t ex_per_phase;        /* S: explicit site potentials per phase, 0..2*CIPHER_MAXCP;
                                    layout.ex_size must be pf_size*S */
    cipher_state_layout layout;  /* offsets of the state planes (see above); map_planes 0 or P */
    int32_t npf;                 /* phases of the problem: a set holding an id >= npf is a bad set */
    int32_t ncp, nmat;           /* components and materials (read when S > 0) */
    /* device copies of the problem's material[nmat] and phasematerialmapping[npf]
     * (in memory the caller owns); required when S > 0, NULL otherwise.  A phase
     * that joins a cell gets SitepotentialExplicit(c0, T of the cell) from them,
     * exactly as cipher_poststep does. */
    const cipher_material *materials;
    const int32_t *phasematerialmapping;
} cipher_grid_desc;

/* The per-step active-set update of cipher_poststep for callers that cannot
 * allocate device memory (an embedding application that owns the device
 * heap, a service with a fixed footprint, code where allocation after
 * start-up is forbidden).  No counterpart in the reference: CIPHER's PostStep
 * allocates its work vectors through PETSc.  Needs no context and calls no
 * allocator; its scratch is a fixed 8 MiB device array inside the library,
 * so grids with (P+1)*stride above 4 Mi entries are rejected (CIPHER_E_ARG).
 * The first call on a device looks the array up with that device current;
 * make that first call before any stream capture.  `stream` must belong to
 * the current device (CIPHER_E_ARG otherwise).  Calls that overlap on the GPU
 * share the array and race.  Synchronises `stream`; returns CIPHER_E_CAP when
 * a superset exceeds P and CIPHER_E_ARG for a bad set in X. */
int cipher_poststep_noalloc(const cipher_grid_desc *g, void *X, void *stream);

/* Y = X + a*F on the PF, DP, EX and TM planes; AS is copied from X
 * (VecWAXPY on the solution vector).  Y may alias X. */
int cipher_waxpy(cipher_ctx *c, void *Y, const void *X, double a, const void *F, void *stream);

/* ------------------------------------------------------------------ */
/* time stepper on device states                                       */
/* (the reference's PETSc TS: InitializeTS src/cipher.c:1097-1115 and   */
/*  the time loop src/cipher.c:1589-1606)                              */
/* ------------------------------------------------------------------ */

enum { CIPHER_TS_RK1FE = 0,     /* forward Euler, fixed step */
       CIPHER_TS_RK2A = 1,      /* Heun 2 with embedded Euler (PETSc -ts_rk_type 2a, the reference's examples) */
       CIPHER_TS_RK3BS = 2 };   /* Bogacki-Shampine 3(2) */

typedef struct cipher_ts_opts {
    int32_t scheme;          /* CIPHER_TS_* */
    int32_t poststep;        /* 1: cipher_poststep after every accepted step (TSSetPostStep) */
    double dt0, dtmin, dtmax;/* first step and step limits (TSAdaptSetStepLimits) */
    double reltol, abstol;   /* TSSetTolerances */
    int64_t max_steps;       /* accepted steps per solve call; 0 = no limit */
} cipher_ts_opts;

typedef struct cipher_ts_stats {
    int64_t steps, rejected, rhs_calls;
    double t, dt, last_norm; /* time reached, next step size, last weighted error norm */
} cipher_ts_stats;

typedef struct cipher_ts cipher_ts;
struct cipher_nucleation;

/* options from the problem: scheme 2a, PostStep on, dt0 = timestep0,
 * limits mintimestep/maxtimestep, tolerances reltol/abstol */
int cipher_ts_default_opts(const cipher_problem *p, cipher_ts_opts *o);
/* stage and candidate buffers are allocated here (ns+1 state vectors) */
int cipher_ts_create(cipher_ctx *c, const cipher_ts_opts *o, cipher_ts **out);
void cipher_ts_destroy(cipher_ts *ts);
/* one attempted step of X from the stepper's time, shortened to end at
 * t_end (TS_EXACTFINALTIME_MATCHSTEP); *accepted tells whether X advanced.
 * Synchronises `stream` (the error norm decides acceptance on the host). */
int cipher_ts_step(cipher_ts *ts, void *X, double t_end, int *accepted, void *stream);
/* steps X from t0 to t_end (or max_steps accepted steps); the step size
 * carries over between calls as the reference's solparams.timestep does */
int cipher_ts_solve(cipher_ts *ts, void *X, double t0, double t_end, cipher_ts_stats *stats, void *stream);
int cipher_ts_get_stats(const cipher_ts *ts, cipher_ts_stats *st);
/* next step size (clamped to the limits); resets the controller history */
int cipher_ts_set_dt(cipher_ts *ts, double dt);
/* run nucleation (before the active-set update) after every accepted step;
 * a firing restarts the step size from dtmin as the reference does
 * (src/cipher.c:861).  NULL detaches. */
int cipher_ts_set_nucleation(cipher_ts *ts, struct cipher_nucleation *nu);

/* ------------------------------------------------------------------ */
/* time stepping with adaptive refinement (the reference's main loop     */
/* with AMR, src/cipher.c:1365-1606 and 1607-1829)                      */
/* ------------------------------------------------------------------ */

typedef struct cipher_amr_opts {
    int32_t nblocks[3];          /* forest blocks per direction (the brick of the reference's forest) */
    int32_t lmin, lmax;          /* minnrefine / maxnrefine; lmax is the voxel grid's level */
    int32_t initcoarsen;         /* adaptations of the initial state (initcoarsen) */
    int32_t interval;            /* accepted steps between adaptations (amrinterval) */
    int32_t precision, device;
    cipher_ts_opts ts;           /* stepper options (max_steps is replaced by interval) */
} cipher_amr_opts;

typedef struct cipher_amr cipher_amr;

/* the forest at the finest level, the SetUpProblem state (chemistry from c0
 * on the device), `initcoarsen` adaptations by the reference's marks, then
 * a device context and stepper over the adapted mesh.  p must outlive it. */
int cipher_amr_create(const cipher_problem *p, const cipher_amr_opts *o, cipher_amr **out);
void cipher_amr_destroy(cipher_amr *a);
/* step to t_end (or max_steps accepted steps, 0 = no limit), adapting
 * every `interval` accepted steps; stats accumulate over the adaptations */
int cipher_amr_solve(cipher_amr *a, double t_end, int64_t max_steps, cipher_ts_stats *stats);
/* the current context, device state, mesh and number of adaptations so far */
int cipher_amr_state(const cipher_amr *a, cipher_ctx **ctx, void **X, const cipher_mesh **m, int64_t *adaptations);

/* ------------------------------------------------------------------ */
/* many independent domains stepped together                           */
/* (no counterpart in the reference, which runs one domain per job)    */
/* ------------------------------------------------------------------ */

enum { CIPHER_BATCH_RUNNING = 0, CIPHER_BATCH_FINISHED = 1, CIPHER_BATCH_FAILED = 2 };

typedef struct cipher_batch cipher_batch;

/* a batch of domains of one precision and dimension on `device`, stepped
 * with the options `o` (each domain with its own step size and error
 * control, exactly as cipher_ts steps it alone) */
int cipher_batch_create(int device, int precision, const cipher_ts_opts *o, cipher_batch **out);
void cipher_batch_destroy(cipher_batch *b);
/* device bytes a domain of context c takes in the batch besides its state */
int cipher_batch_footprint(const cipher_batch *b, const cipher_ctx *c, int64_t *bytes);
/* add the domain of context c with device state X (the caller keeps both
 * alive until detach), to be stepped from t0 to t_end; allocates the
 * domain's stage buffers.  Membership changes rebuild the batch's launch
 * tables, tile shapes (timed once per domain class) and CUDA graph. */
int cipher_batch_attach(cipher_batch *b, cipher_ctx *c, void *X, double t0, double t_end, int *slot);
/* remove a domain; its X is brought up to date first */
int cipher_batch_detach(cipher_batch *b, int slot);
/* one attempted step of every running domain (one graph launch, one host
 * synchronisation); *running = domains that have not reached t_end.  A
 * domain's X is current after cipher_batch_flush, detach, or once no
 * domain runs; a failed domain (cap overflow, bad set, non-finite error)
 * stops and reports its code through cipher_batch_slot_stats. */
int cipher_batch_step(cipher_batch *b, int *running);
int cipher_batch_flush(cipher_batch *b);
int cipher_batch_slot_stats(const cipher_batch *b, int slot, cipher_ts_stats *st, int *status, int *error);
/* 1 (default): replay each step from a CUDA graph; 0: launch directly */
int cipher_batch_set_graphs(cipher_batch *b, int on);
/* launch-table rebuilds, and steps replayed from a graph or launched directly */
int cipher_batch_get_counters(const cipher_batch *b, int64_t *rebuilds, int64_t *graph_steps, int64_t *direct_steps);

/* ------------------------------------------------------------------ */
/* serving: continuous batching of many simulations on one GPU          */
/* (no counterpart in the reference)                                   */
/* ------------------------------------------------------------------ */

enum { CIPHER_INIT_SHARP = 0,     /* SetUpProblem state (+ chemistry from c0) */
       CIPHER_INIT_DIFFUSE = 1 }; /* diffuse Voronoi state of the given width */

typedef struct cipher_server_opts {
    int32_t device, precision;
    int32_t max_active;          /* domains stepped together at most */
    int64_t hbm_budget;          /* device bytes the admitted requests may hold */
    cipher_ts_opts ts;           /* stepper options of every request */
} cipher_server_opts;

typedef struct cipher_server_result_t {
    int32_t state;               /* 0 queued, 1 running, 2 done */
    int32_t status, error;       /* CIPHER_BATCH_* and the error code of a failed request */
    cipher_ts_stats stats;
    double t_submit, t_admit, t_finish;  /* CLOCK_MONOTONIC seconds */
    int64_t ncells;
    int32_t ndof;
    int64_t footprint;           /* device bytes charged against the budget */
} cipher_server_result_t;

typedef struct cipher_server cipher_server;

int cipher_server_create(const cipher_server_opts *o, cipher_server **out);
void cipher_server_destroy(cipher_server *s);
/* queue a request; the server takes ownership of p (freed on release or
 * destroy) and builds its mesh, context and initial state on admission */
int cipher_server_submit(cipher_server *s, cipher_problem *p, int init_kind, double width, double t_end, int64_t *id);
/* admit queued requests in arrival order while they fit the budget, take
 * one batched step of every running request, retire the finished ones
 * (their final state is copied to host memory and their device memory
 * freed) */
int cipher_server_poll(cipher_server *s, int *queued, int *active, int *done);
/* a request's state and timings; X (ncells x ndof doubles, reference AoS
 * layout) receives the final state of a finished request when not NULL */
int cipher_server_result(const cipher_server *s, int64_t id, cipher_server_result_t *res, double *X);
int cipher_server_release(cipher_server *s, int64_t id);
/* device bytes held by admitted requests now and at most so far */
int cipher_server_usage(const cipher_server *s, int64_t *used, int64_t *peak);

/* where a server's host time goes */
typedef struct cipher_server_counters {
    int64_t polls, steps, domain_steps;      /* batch steps, and domains stepped in them */
    int64_t rebuilds, graph_steps, direct_steps;
    double t_admit, t_step, t_retire;        /* seconds in each phase of cipher_server_poll */
} cipher_server_counters;
int cipher_server_get_counters(const cipher_server *s, cipher_server_counters *c);

/* ------------------------------------------------------------------ */
/* nucleation (the first part of PostStep, src/cipher.c:715-867;        */
/* models src/material.c:47-290)                                       */
/* ------------------------------------------------------------------ */

/* same numbering as nucleation_model_t (src/typedef.h:45-51) */
enum { CIPHER_NUC_CNT = 0, CIPHER_NUC_CONSTANT = 1, CIPHER_NUC_THERMAL = 2, CIPHER_NUC_NONE = 3 };

typedef struct cipher_nucleus {
    int32_t model;
    int32_t nmatrix;
    int32_t matrix[16];                  /* sorted phase ids a site's cells may hold */
    int8_t active_solutes[CIPHER_MAXCP];
    double gamma, shapefactor, minsize, atomicvolume, lengthscale;   /* cnt and thermal */
    double incubationtimemin, liquidus;
    double nucleation_rate;                                          /* constant */
    double solvus_temperature_0, enthalpy_fusion_0;                  /* thermal */
    int32_t has_solvus_c, has_enthalpy_c;
    double solvus_temperature_c[CIPHER_MAXCP], enthalpy_fusion_c[CIPHER_MAXCP];
} cipher_nucleus;

typedef struct cipher_nucleation cipher_nucleation;

/* nucleation sites of context c: voxelsite[cell] = the cell's site or -1,
 * sitephase/sitenucleus per site, the nuclei's parameters, and the seed of
 * the event draws (the reference draws with rand(); here a splitmix64
 * stream per object, so runs are reproducible) */
int cipher_nucleation_create(cipher_ctx *c, int nsites, const int32_t *voxelsite, const int32_t *sitephase,
                             const int32_t *sitenucleus, int nnuclei, const cipher_nucleus *nuclei, uint64_t seed,
                             cipher_nucleation **out);
void cipher_nucleation_destroy(cipher_nucleation *nu);
/* one nucleation update of X at time t after a step of size dt: a site
 * whose cells hold a phase outside its nucleus' matrix is retired; every
 * other active site averages the barrier, diffusivity and temperature over
 * its cells and draws its event; fired sites turn into their phase (set,
 * phi, explicit potentials of c0) and are retired.  *nfired = sites fired
 * (the reference then restarts the stepper from mintimestep).  Synchronises
 * `stream`.  The active-set update (cipher_poststep) follows. */
int cipher_nucleation_step(cipher_nucleation *nu, void *X, double t, double dt, int *nfired, void *stream);
/* per site: 1 active, 0 retired; and the last averages (NaN when unset) */
int cipher_nucleation_sites(const cipher_nucleation *nu, int8_t *active, double *barrier, double *diffusivity,
                            double *temperature, double *volume);

/* ------------------------------------------------------------------ */
/* output (the reference's output step in PostStep, src/cipher.c:976-1093) */
/* ------------------------------------------------------------------ */

enum { CIPHER_OUT_PHASEID = 0,      /* id of the phase with the largest interpolant */
       CIPHER_OUT_MATID = 1,        /* its material */
       CIPHER_OUT_INTERFACEID = 2,  /* interface of the cell's last phase pair, -1 for one phase */
       CIPHER_OUT_CHEMPOT = 3,      /* mu of component `index` (0 for the last component) */
       CIPHER_OUT_COMP = 4,         /* interpolated composition of component `index` */
       CIPHER_OUT_PHI = 5,          /* phase fraction of phase `index` (0 where inactive) */
       CIPHER_OUT_TEMPERATURE = 6 };

typedef struct cipher_output_field {
    int32_t kind, index;
    char name[48];               /* array name in the output file */
} cipher_output_field;

/* derived fields of device state X into the device array out[nfields][ncells] */
int cipher_output_fields(cipher_ctx *c, const void *X, const cipher_output_field *fields, int nfields, double *out,
                         void *stream);
/* a VTK XML unstructured-grid file (.vtu, raw appended data) of the uniform
 * grid of p with cell-data arrays values[nfields][ncells] (host) */
int cipher_write_vtu(const char *path, const cipher_problem *p, const cipher_output_field *fields, int nfields,
                     const double *values);

/* reference AoS layout (ncells x ndof doubles, device) <-> device state */
int cipher_state_from_aos(cipher_ctx *c, const double *aos, void *X, void *stream);
int cipher_state_to_aos(cipher_ctx *c, const void *X, double *aos, void *stream);

/* drop-in call with HOST buffers in the reference AoS layout: copies X to the
 * device, evaluates the RHS and copies F back (synchronous on `stream`;
 * RHSFunction, src/cipher.c:27).  3D phase-field grids of four or more
 * planes go through in z-slabs on the context's own streams, so that copies
 * out overlap copies in; pinned host buffers give full copy speed. */
int cipher_rhs_aos_host(cipher_ctx *c, double t, const double *X_host, double *F_host, void *stream);

/* ------------------------------------------------------------------ */
/* configuration files (the reference's YAML input, SetUpConfig,        */
/* src/init.c:24-1716)                                                  */
/* ------------------------------------------------------------------ */

/* everything a configuration file sets: the problem, nucleation, output
 * fields, and the solver / AMR / output parameters the problem does not hold */
typedef struct cipher_config {
    cipher_problem *problem;              /* owned; voxelphase from voxel_phase_mapping */
    int32_t ncomponents;
    char componentname[CIPHER_MAXCP][64];
    /* nucleation: header n_sites / nuclei, nucleus/<name>, site mappings */
    int32_t nsites, nnuclei;
    int32_t *voxelsite;                   /* [prod(resolution)] site of each voxel, -1 for none; NULL without sites */
    int32_t *sitephase, *sitenucleus;     /* [nsites] */
    cipher_nucleus *nuclei;               /* [nnuclei] */
    /* output fields (header outputs) and their cadence */
    int32_t noutputs;
    cipher_output_field *outputs;         /* [noutputs] */
    int32_t outputfreq;
    char outfile[256];
    /* stepper and mesh parameters (solution_parameters) */
    char petscoptions[1024];
    char rk_type[16];                     /* -ts_rk_type of petscoptions, else PETSc's default "3bs" */
    int32_t has_random_seed;
    int64_t random_seed;
    int32_t initblocksize[3], initrefine, initcoarsen, maxnrefine, minnrefine, amrinterval;
    int32_t max_phase_neighbours;
} cipher_config;

/* parse a configuration held in memory; `basedir` (or NULL) is where
 * mapping files named "*.txt" are looked for first (then the working
 * directory, as the reference does).  Errors name the property at fault. */
int cipher_config_parse(const char *text, size_t len, const char *basedir, cipher_config **out);
/* read and parse a configuration file */
int cipher_config_load(const char *path, cipher_config **out);
void cipher_config_free(cipher_config *c);
/* one output name of the configuration format ("phaseid", "matid",
 * "interfaceid", "temperature", "<comp>_chempot", "<comp>_c", "<phase>_phi")
 * as a field, read as the reference's output step reads it (src/cipher.c:
 * 1005-1080); a component that is not listed gives a zero field */
int cipher_output_field_parse(const char *name, int ncomponents, const char *const *components,
                              cipher_output_field *out);
/* the configuration parser's view of a YAML text as JSON (objects, arrays,
 * strings), for checking a file; *needed = bytes including the final NUL */
int cipher_yaml_to_json(const char *text, size_t len, char *out, size_t outlen, size_t *needed);

#ifdef __cplusplus
}
#endif
#endif /* CIPHER_B200_H */
