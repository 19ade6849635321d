/*
 * cipher_problem.h - host-side description of a CIPHER phase-field problem.
 *
 * Plain C structs (no CUDA, no torch) holding the model parameters, the
 * finite-volume leaf mesh and the per-cell state layout that the reference
 * keeps in its AppCtx (src/typedef.h:145-319) and DMPlex section
 * (src/cipher.c:1162-1172, src/init.c:1330-1343).
 *
 * The tables are fixed-capacity and stored inline so that a problem can be
 * copied, serialised and flattened to device tables without pointer chasing.
 * Table orderings follow the reference parser exactly (src/init.c), so that a
 * table index in this file is the same index the reference's model code walks
 * with its `currentbinary++` / `currentternary++` pointers (src/material.c).
 */
#ifndef CIPHER_PROBLEM_H
#define CIPHER_PROBLEM_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CIPHER_MAXCP     5    /* max components           (src/typedef.h:28) */
#define CIPHER_MAXAP     15   /* default active-set cap    (src/typedef.h:29) */
#define CIPHER_MAXTSER   10   /* terms in a T-series      (src/typedef.h:147) */
#define CIPHER_MAXRK     4    /* Redlich-Kister orders kept per pair */
#define CIPHER_MAXRKTAB  50   /* C(5,2)*5 = C(5,3)*5 = 50 pair/triple tables */
#define CIPHER_MAXBIN    10   /* C(5,2) */
#define CIPHER_MAXSRC    2    /* sources per material / interface */
#define CIPHER_MAXDIR    8    /* anisotropy directions */
#define CIPHER_MAXLC     64   /* load cases */
#define CIPHER_MAXBC     6    /* boundary conditions (src/init.c: assert <= 6) */

#define CIPHER_TOL       1.0e-6     /* src/typedef.h:26 */
#define CIPHER_LARGE     1.0e+6     /* src/typedef.h:25 */
#define CIPHER_R_GAS     8.314462   /* src/typedef.h:30 */

/* chemical free-energy model; same numbering as chemfe_model_t (src/typedef.h:54-59) */
enum { CIPHER_CHEM_QUADRATIC = 0, CIPHER_CHEM_CALPHADDIS = 1,
       CIPHER_CHEM_CALPHAD2SL = 2, CIPHER_CHEM_NONE = 3 };
/* interpolation; same numbering as interpolation_t (src/typedef.h:69-74) */
enum { CIPHER_INTERP_LINEAR = 0, CIPHER_INTERP_QUADRATIC = 1, CIPHER_INTERP_CUBIC = 2 };
/* boundary type; same numbering as boundary_t (src/typedef.h:62-66) */
enum { CIPHER_BC_NEUMANN = 0, CIPHER_BC_DIRICHLET = 1, CIPHER_BC_NONE = 2 };
/* source model; same numbering as source_model_t (src/typedef.h:40-43) */
enum { CIPHER_SOURCE_SINK = 0, CIPHER_SOURCE_RANDOM = 1 };

/* sum_i coeff[i]*T^exp[i] + logcoeff*T*ln(T)   (TSeries, src/typedef.h:145-150) */
typedef struct cipher_tseries {
    int32_t n;
    int32_t exp[CIPHER_MAXTSER];
    double  coeff[CIPHER_MAXTSER];
    double  logcoeff;
} cipher_tseries;

/* Redlich-Kister expansion of one pair / triple (RK, src/typedef.h:153-156);
 * i[] is the ternary component index used by the calphaddis model. */
typedef struct cipher_rk {
    int32_t n;
    int32_t i[CIPHER_MAXRK];
    cipher_tseries h[CIPHER_MAXRK];
} cipher_rk;

/* component mobility (TACTIVATIONPROP, src/typedef.h:159-163) */
typedef struct cipher_mobility {
    double m0;
    cipher_tseries unary[CIPHER_MAXCP];      /* migration energy per component */
    cipher_rk binary[CIPHER_MAXBIN];         /* C(ncp,2), order (cj<ci) */
} cipher_mobility;

/* solute source (SOURCE, src/typedef.h:77-96) */
typedef struct cipher_source {
    int32_t model;                           /* CIPHER_SOURCE_* */
    double rate[CIPHER_MAXCP], ceq[CIPHER_MAXCP], amplitude[CIPHER_MAXCP];
} cipher_source;

/* phase material (MATERIAL, src/typedef.h:210-218 with CHEMFE/THERMAL) */
typedef struct cipher_material {
    int32_t model;                           /* CIPHER_CHEM_* */
    int32_t nsites;                          /* 0 none, 1 quadratic/calphaddis, 2 calphad2sl */
    double  molarvolume;
    double  chempot_ex_kineticcoeff;
    double  c0[2 * CIPHER_MAXCP];            /* [nsites*ncp] */
    double  stoichiometry[2];                /* [nsites] */
    double  p, q;                            /* calphad2sl sublattice ratios */
    cipher_tseries ref;                      /* none / quadratic / calphaddis reference energy */
    /* quadratic & calphaddis: unary[ncp]; calphad2sl: unary[cp*ncp+cq] */
    cipher_tseries unary[CIPHER_MAXCP * CIPHER_MAXCP];
    cipher_tseries quad_ceq[CIPHER_MAXCP];   /* quadratic */
    cipher_tseries quad_binary[CIPHER_MAXCP];/* quadratic */
    /* calphaddis: binary C(ncp,2), ternary C(ncp,3)
     * calphad2sl: binary = binaryp [(cp_i<cp_j), cq], ternary = ternaryp [(i<j<k), cq],
     *             binaryq [cp, (cq_i<cq_j)], ternaryq [cp, (i<j<k)] */
    cipher_rk binary[CIPHER_MAXRKTAB];
    cipher_rk ternary[CIPHER_MAXRKTAB];
    cipher_rk binaryq[CIPHER_MAXRKTAB];
    cipher_rk ternaryq[CIPHER_MAXRKTAB];
    cipher_mobility mobilityc[CIPHER_MAXCP];
    /* thermal (THERMAL, src/typedef.h:204-207) */
    double  temperature0;
    cipher_tseries specific_heat, latent_heat, tconductivity;
    /* bulk sources */
    int32_t nsources;
    cipher_source sources[CIPHER_MAXSRC];
} cipher_material;

/* interface (INTERFACE/IENERGY/IMOBILITY, src/typedef.h:221-240) */
typedef struct cipher_interface {
    double  width;
    double  energy_m0;                       /* ienergy->e->m0 */
    cipher_tseries energy_activation;        /* ienergy->e->unary[0] */
    int32_t energy_naniso;
    double  energy_aniso_dir[CIPHER_MAXDIR * 3], energy_aniso_val[CIPHER_MAXDIR];
    double  mobility_m0;                     /* imobility->m->m0 */
    cipher_tseries mobility_activation;      /* imobility->m->unary[0] */
    int32_t mobility_naniso;
    double  mobility_aniso_dir[CIPHER_MAXDIR * 3], mobility_aniso_val[CIPHER_MAXDIR];
    int32_t has_potential;                   /* segregation potential present */
    double  potential[CIPHER_MAXCP];         /* [ndp] */
    int32_t has_mobilityc;                   /* interface solute mobility present */
    double  mobilityc[CIPHER_MAXCP];         /* [ncp] */
    int32_t nsources;
    cipher_source sources[CIPHER_MAXSRC];
} cipher_interface;

/* boundary condition (BOUNDARYCONDITIONS, src/typedef.h:243-248) */
typedef struct cipher_bc {
    int32_t boundaryid;                      /* face label 1..2*dim */
    int32_t chem_bctype, thermal_bctype;     /* CIPHER_BC_* */
    double  chem_bcval[CIPHER_MAXCP];
    double  thermal_bcval;
    int8_t  chem_bcbool[CIPHER_MAXCP];
} cipher_bc;

/* model + solver parameters (AppCtx minus mesh, src/typedef.h:277-319) */
typedef struct cipher_problem {
    int32_t dim;
    int32_t npf, ncp, ndp, nmat, nf, nbcs;
    int32_t pf_size;            /* P  = min(max_phase_neighbours, npf)  (src/init.c:1336) */
    int32_t maxsites;           /* max nsites over materials             (src/init.c:~868) */
    int32_t interpolation;      /* CIPHER_INTERP_* */
    int32_t gradient_calculation;
    double  junctionpenalty;
    int32_t nloadcases, currentloadcase, has_temperature_rate;
    double  time[CIPHER_MAXLC], temperature_rate[CIPHER_MAXLC];
    double  timestep0, mintimestep, maxtimestep, reltol, abstol;
    int32_t resolution[3];
    double  size[3];
    int32_t periodic[3];
    cipher_material  *material;            /* [nmat] */
    cipher_interface *interface;           /* [nf]   */
    int32_t *interfacelist;                /* [npf*npf], pair (a<b) at a*npf+b */
    int32_t *phasematerialmapping;         /* [npf] */
    int32_t *voxelphase;                   /* [prod(resolution)] initial phase per voxel, x fastest */
    cipher_bc bcs[CIPHER_MAXBC];
    double  *centres;                      /* [npf*3] grain centres of Voronoi maps, or NULL */
} cipher_problem;

/*
 * Finite-volume leaf mesh, linearised.
 *
 * Cells [0, nowned) are owned, [nowned, ncells) are ghosts (a one-cell halo).
 * Interior faces are listed in face order; the reference accumulates face
 * fluxes in exactly this order (src/cipher.c:236-317).  face_cells[2f] is the
 * support cell L and face_cells[2f+1] is R.  Boundary faces (support size 1)
 * carry the label 1..2*dim the reference assigns from the face centroid
 * (src/cipher.c:1209-1221).
 */
typedef struct cipher_mesh {
    int32_t dim;
    int32_t ncells, nowned;
    int32_t nfaces;
    int32_t *face_cells;        /* [2*nfaces] */
    int32_t nbfaces;
    int32_t *bface_cell;        /* [nbfaces] */
    int32_t *bface_label;       /* [nbfaces] */
    double  *cellgeom;          /* [ncells] delta = vol^(1/dim) (src/cipher.c:1226-1230) */
    int32_t *cell_global;       /* [ncells] index of the cell in the full grid */
    /* uniform grid description (all meshes built by cipher_mesh_uniform) */
    int32_t uniform;
    int32_t res[3];
    int32_t periodic[3];
    int32_t slab_lo, slab_hi;   /* owned slab [lo,hi) along the slowest axis */
} cipher_mesh;

/* reference per-cell dof layout, all doubles: [AS P+1 | PF P | DP D | EX P*S | TM 1] */
typedef struct cipher_aos_layout {
    int32_t as_offset, pf_offset, dp_offset, ex_offset, tm_offset, ndof;
    int32_t as_size, pf_size, dp_size, ex_size, sp_size, sf_size;
} cipher_aos_layout;

#ifdef __cplusplus
}
#endif
#endif /* CIPHER_PROBLEM_H */
