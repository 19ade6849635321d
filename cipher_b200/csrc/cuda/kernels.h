/*
 * kernels.h - launch interfaces of the device kernels (internal to the
 * library; the public C ABI is include/cipher_b200.h).
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"

namespace cipher {

/* long-lived device buffers from a per-device stream-ordered pool
 * (devmem.cu): dev_alloc's memory is usable on any stream when it returns;
 * dev_free does not wait, so no queued work may still use the block */
cudaError_t dev_alloc(void **ptr, size_t bytes);
void dev_free(void *ptr);
template <typename T>
inline cudaError_t dev_alloc(T **ptr, size_t bytes) { return dev_alloc((void **)ptr, bytes); }
/* a pinned host slot of up to 64 bytes (zeroed), for small device-to-host results */
cudaError_t pinned_word_alloc(void **ptr);
void pinned_word_free(void *ptr);
template <typename T>
inline cudaError_t pinned_word_alloc(T **ptr) { return pinned_word_alloc((void **)ptr); }

/* the faces of a non-uniform (adapted) mesh, per cell: entries
 * [start[c], start[c+1]) list cell c's faces in the reference's face order
 * (the order of the mesh's face list).  start == NULL: a uniform grid whose
 * faces follow from res/per. */
struct FaceLists {
    const int32_t *start;        /* [ncells+1] */
    const int32_t *nbr;          /* [nnz] the other cell of the face; bit 31 set when c is the face's L cell */
    const int32_t *face;         /* [nnz] face index */
    const double *ff;            /* [nfaces] 2*(vol/delta of the smaller cell)/(delta_L+delta_R) (src/cipher.c:273-275) */
    const double *vol, *delta;   /* [ncells] delta^dim and cellgeom */
    const int32_t *bstart;       /* [ncells+1] boundary faces of each cell */
    const int32_t *blabel;       /* their labels 1..2*dim */
};
constexpr int32_t FACE_SELF_L = (int32_t)0x80000000u;

/* classes of the kernels' cell grouping (general kernels: one per material
 * for single-phase cells, then sets of 2, 3 and more phases; FP64 phase-field
 * kernel: the set size) */
constexpr int kOrderClasses = 32;

/* arguments of the phase-field-only RHS on a uniform grid */
template <typename R>
struct PfArgs {
    int64_t ncells, stride;
    int res[3];
    int per[3];
    int P, npf;
    double ffactor, vol;          /* face factor and cell volume (src/cipher.c:273-275) */
    int geom_mode;                /* GEOM_DIVIDE / GEOM_RECIP / GEOM_UNIT (pf_gather.cuh) */
    double inv_vol;               /* 1/vol, exact when vol is a power of two */
    double face_coef;             /* ffactor/vol, for the mixed path */
    double junctionpenalty;
    int has_temp_rate;
    double temp_rate;
    int single;                   /* every pair uses one T-independent interface */
    int zbase, zcount;            /* planes [zbase, zbase+zcount) of a 3D grid; zcount 0 = all */
    double sig0, mob0, wid0, tj0; /* its sigma, m, w and triple-junction weight */
    /* FP32 forms for the mixed single-interface kernel: sigma, 1/w, w/pi^2,
     * tj/2, m and ffactor/vol; thresholds such that for a float p the float
     * tests p > tol_gt, p < tol1_lt, p < tol_lt, p > tol1_gt equal the double
     * tests p > TOL, p < 1-TOL, p < TOL, p > 1-TOL */
    float sig_f, inv_w_f, w_pi2_f, tjh_f, mob_f, coef_f;
    float tol_gt, tol1_lt, tol_lt, tol1_gt;
    const int32_t *itflist;
    const DevInterface *itfs;
    const uint16_t *as;
    const uint32_t *maps;         /* [P][stride] face maps: one word per slot (cipher_b200.h) */
    const R *phi;
    const R *tm;
    R *fphi;
    R *ftm;
    int *err;
    /* FP64 reference-order kernel: cells grouped by set size (NULL: grid order) */
    int32_t *order;               /* [ncells] */
    int32_t *order_cursor;        /* [kOrderClasses] class totals */
    int32_t *order_counts;        /* [kOrderClasses][blocks of 256 cells] */
};

cudaError_t launch_rhs_phasefield(const PfArgs<double> &a, int dim, cudaStream_t s);
/* the closed-form single-interface kernel in FP64 (rhs_mixed.cu) */
cudaError_t launch_rhs_items_fp64(const PfArgs<double> &a, int dim, cudaStream_t s);
cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s);

/* many independent domains in one launch: domain i owns tiles
 * [tile_start[i], tile_start[i+1]) of the global tile list; a tile is
 * BX x BY cells of one (y, z) row range of that domain */
template <typename R>
struct BatchTiles {
    const PfArgs<R> *args;        /* [n] device */
    const int64_t *tile_start;    /* [n+1] device */
    const int *active;            /* [n] device: 0 skips the domain */
    int n;
    int64_t total;                /* tile_start[n] */
    int pmax;                     /* largest P of the batch (shared-memory columns) */
    int i32;                      /* every member's plane offsets fit 32-bit indices */
};

/* grid: persistent (a multiple of the SM count); by = tile rows (1, 2, 4) */
cudaError_t launch_rhs_pf_batched(const BatchTiles<double> &b, int dim, int single, int by, int grid, cudaStream_t s);
cudaError_t launch_rhs_pf_batched(const BatchTiles<float> &b, int dim, int single, int by, int grid, cudaStream_t s);

/* one boundary condition, flattened (BOUNDARYCONDITIONS, src/typedef.h:243-248) */
struct DevBC {
    int label, chem_type, thermal_type;
    double chem_val[CIPHER_MAXCP];
    int chem_on[CIPHER_MAXCP];
    double thermal_val;
};

/* arguments of the general RHS on a uniform grid: chemistry, heat,
 * boundary faces, several interfaces and materials */
template <typename R>
struct GenArgs {
    int64_t ncells, stride;
    int res[3];
    int per[3];
    int P, npf, ncp, ndp, SP;     /* SP = site potentials per phase (maxsites*ndp) */
    int interp;
    double ffactor, vol, inv_vol;
    int geom_mode;
    double delta;                 /* cell size (cellgeom) */
    double junctionpenalty;
    int has_temp_rate;
    double temp_rate;
    const int32_t *itflist;
    const DevInterface *itfs;
    ChemTables chem;
    int nbcs;
    DevBC bcs[CIPHER_MAXBC];
    const uint16_t *as;
    const R *phi;
    const double *dp;
    const double *ex;
    const R *tm;
    double *comp, *mob, *tcond;   /* per-cell scratch: [ncp][stride], [ncp][stride], [stride] */
    FaceLists fl;                 /* face lists of an adapted mesh (fl.start == NULL: uniform grid) */
    double *grad;                 /* [dim][P][stride] phase-field gradients, or NULL (no anisotropy) */
    int32_t *order;               /* [ncells] cells grouped by class (single-phase material, set size), or NULL */
    int32_t *order_cursor;        /* [kOrderClasses] class totals of the grouping */
    int32_t *order_counts;        /* [kOrderClasses][blocks of 256 cells] per-block counts, then offsets */
    int nclass;                   /* classes in use: nmat + 3 (0: no grouping) */
    uint32_t single_models;       /* bit m: single-phase cells of model m run in rhs_single.cu's kernels */
    double *iscr;                 /* [ItemQ::nq][icap] model results of the (cell, phase) items (rhs_items.cu) */
    int32_t *ibase;               /* [ncells] first item of a cell of several phases, or -1 (no items) */
    int32_t *icell;               /* [icap] item -> cell * 16 + slot */
    int32_t *icount;              /* [1] items asked for by this RHS (may exceed icap) */
    int64_t icap;                 /* item capacity (0: no item path) */
    int item_model;               /* >= 0: every material has this model (items compiled for it), else -1 */
    double cw[3];                 /* cell width along each axis: centroid = (i + 0.5) * cw */
    R *fphi;
    double *fdp, *fex;
    R *ftm;
    int *err;
};

/* nucleation (rhs_general.cu): cells of site s are list[start[s] .. start[s+1]) */
struct NucArgs {
    int nsites, ncp_stride;               /* per-cell record: 3 + ncp doubles */
    const int32_t *list;                  /* cells sorted by site */
    const int64_t *start;                 /* [nsites+1] */
    const int32_t *site_of;               /* [nlist] site of each listed cell */
    const int32_t *sitephase, *sitenucleus;
    const cipher_nucleus *nuclei;
    const int8_t *active;                 /* [nsites] */
    double *cellrec;                      /* [nlist][3 + ncp]: ok, barrier, T, diffusivity[ncp] */
    double *siterec;                      /* [nsites][4 + ncp]: ok, volume, T*vol, barrier*vol, diff*vol[ncp] */
    const int8_t *fired;                  /* [nsites] */
    double vol;
};
cudaError_t launch_nucleation_sums(const GenArgs<double> &a, const NucArgs &n, int64_t nlist, cudaStream_t s);
cudaError_t launch_nucleation_sums(const GenArgs<float> &a, const NucArgs &n, int64_t nlist, cudaStream_t s);
cudaError_t launch_nucleation_reset(const GenArgs<double> &a, const NucArgs &n, int64_t nlist, cudaStream_t s);
cudaError_t launch_nucleation_reset(const GenArgs<float> &a, const NucArgs &n, int64_t nlist, cudaStream_t s);

/* output fields of a state (rhs_general.cu); fields are the public
 * cipher_output_field descriptors in device memory */
cudaError_t launch_output_fields(const GenArgs<double> &a, const int32_t *kinds, const int32_t *idx, int nf,
                                 double *out, cudaStream_t s);
cudaError_t launch_output_fields(const GenArgs<float> &a, const int32_t *kinds, const int32_t *idx, int nf,
                                 double *out, cudaStream_t s);
cudaError_t launch_rhs_general(const GenArgs<double> &a, int dim, cudaStream_t s);
cudaError_t launch_rhs_general(const GenArgs<float> &a, int dim, cudaStream_t s);
/* the single-phase cells of the models in a.single_models (rhs_single.cu):
 * their composition, mobility and conductivity, then their RHS */
cudaError_t launch_chem_single(const GenArgs<double> &a, cudaStream_t s);
cudaError_t launch_chem_single(const GenArgs<float> &a, cudaStream_t s);
cudaError_t launch_rhs_single(const GenArgs<double> &a, int dim, cudaStream_t s);
cudaError_t launch_rhs_single(const GenArgs<float> &a, int dim, cudaStream_t s);
/* the (cell, phase) items of the cells of several phases (rhs_items.cu):
 * list them (a.ibase, a.icell), then evaluate each phase's models into the
 * item scratch; a.icap > 0 */
cudaError_t launch_items(const GenArgs<double> &a, cudaStream_t s);
cudaError_t launch_items(const GenArgs<float> &a, cudaStream_t s);
/* EX of every listed phase and mu of the majority phase from the materials'
 * c0 at the cell temperature (src/init.c:1790-1823) */
cudaError_t launch_chem_init(const GenArgs<double> &a, double *ex, double *dp, cudaStream_t s);
cudaError_t launch_chem_init(const GenArgs<float> &a, double *ex, double *dp, cudaStream_t s);

/* per-step active-set update on a uniform grid (src/cipher.c:869-974) */
template <typename R>
struct PostArgs {
    int64_t ncells, stride;
    int res[3];
    int per[3];
    int P, S;                     /* S = explicit site potentials per phase */
    uint16_t *as;
    R *phi;
    double *ex;
    const R *tm;
    uint16_t *pruned;             /* scratch: pruned sets, [P+1][stride] */
    uint32_t *maps;               /* face maps rebuilt after the union, or NULL */
    int npf;
    ChemTables chem;              /* with chem.mat set, new phases get SitepotentialExplicit(c0, T) */
    FaceLists fl;                 /* neighbours of an adapted mesh (fl.start == NULL: uniform grid) */
    int *err;
};

cudaError_t launch_poststep(const PostArgs<double> &a, int dim, cudaStream_t s);
cudaError_t launch_poststep(const PostArgs<float> &a, int dim, cudaStream_t s);
/* the face maps of a state from its sets (also part of launch_poststep) */
cudaError_t launch_build_maps(const PostArgs<double> &a, int dim, cudaStream_t s);
cudaError_t launch_build_maps(const PostArgs<float> &a, int dim, cudaStream_t s);
/* cells [c0, c1) only */
cudaError_t launch_build_maps_range(const PostArgs<double> &a, int dim, int64_t c0, int64_t c1, cudaStream_t s);
cudaError_t launch_build_maps_range(const PostArgs<float> &a, int dim, int64_t c0, int64_t c1, cudaStream_t s);

/* batched PostStep: domain i owns blocks [block_start[i], block_start[i+1])
 * of 256 cells; domains whose `active` entry is 0 are skipped */
template <typename R>
struct BatchPost {
    const PostArgs<R> *args;      /* [n] device */
    const int64_t *block_start;   /* [n+1] device: blocks of 256 cells (pruning) */
    const int *active;            /* [n] device */
    int n;
    int64_t total;
    const int64_t *row_start;     /* [n+1] device: row blocks (4 rows of 32 cells; union and face maps) */
    int64_t row_total;
    int pmax;                     /* largest P of the batch (shared-memory staging) */
};
/* row blocks of a uniform grid (union and face-map kernels) */
int64_t post_row_blocks(const int *res);
cudaError_t launch_poststep_batched(const BatchPost<double> &b, int dim, cudaStream_t s);
cudaError_t launch_poststep_batched(const BatchPost<float> &b, int dim, cudaStream_t s);

/* reference AoS (ncells x ndof doubles) <-> plane-major device state */
struct LayoutArgs {
    int64_t ncells, stride;
    int P, D, E;                  /* PF slots, DP count, EX count (P*S) */
    int ndof, as_off, pf_off, dp_off, ex_off, tm_off;
    int real_bytes;               /* 8 (FP64) or 4 (mixed) for PF and TM */
    uint16_t *as;
    void *phi;
    double *dp;
    double *ex;
    void *tm;
};
cudaError_t launch_aos_to_soa(const LayoutArgs &a, const double *aos, cudaStream_t s);
/* state of an adapted mesh from the old mesh's state (src0/nsrc: device transfer plan) */
cudaError_t launch_transfer(const LayoutArgs &dst, const LayoutArgs &src, const int64_t *src0, const int32_t *nsrc,
                            cudaStream_t s);
/* cells [c0, c1) of the domain (aos is the whole domain's array) */
cudaError_t launch_aos_to_soa_range(const LayoutArgs &a, const double *aos, int64_t c0, int64_t c1, cudaStream_t s);

/* SetUpProblem state from a device voxel map (layout.cu) */
struct InitArgs {
    LayoutArgs L;
    int res[3], per[3], dim, npf;
    const int32_t *voxel;         /* [ncells] phase per cell */
    const double *t0;             /* [npf] temperature0 of each phase's material */
    int *err;
};
cudaError_t launch_init_sharp(const InitArgs &a, cudaStream_t s);
cudaError_t launch_soa_to_aos(const LayoutArgs &a, double *aos, int include_as, cudaStream_t s);
cudaError_t launch_soa_to_aos_range(const LayoutArgs &a, double *aos, int include_as, int64_t c0, int64_t c1,
                                    cudaStream_t s);

/* what the batch driver needs to know of a context (context.cu) */
struct CtxInfo {
    int device, precision, dim, general, single, P;
    int listed;                   /* an adapted mesh (face lists) */
    int64_t ncells;
    int res[3];
};

}  // namespace cipher

struct cipher_ctx;
namespace cipher {
CtxInfo ctx_info(const cipher_ctx *c);
PfArgs<double> ctx_pf_args_d(const cipher_ctx *c, const void *X, void *F, int *err);
PfArgs<float> ctx_pf_args_f(const cipher_ctx *c, const void *X, void *F, int *err);
PostArgs<double> ctx_post_args_d(const cipher_ctx *c, void *X, uint16_t *pruned, int *err);
PostArgs<float> ctx_post_args_f(const cipher_ctx *c, void *X, uint16_t *pruned, int *err);
cudaError_t ctx_rhs_general(const cipher_ctx *c, const void *X, void *F, int *err, cudaStream_t s);
GenArgs<double> ctx_gen_args_d(const cipher_ctx *c, const void *X);
GenArgs<float> ctx_gen_args_f(const cipher_ctx *c, const void *X);
double ctx_cell_volume(const cipher_ctx *c);
}  // namespace cipher
