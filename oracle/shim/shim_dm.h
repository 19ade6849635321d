/*
 * shim_dm.h - concrete objects behind the PETSc shim handles (oracle only).
 */
#ifndef CIPHER_SHIM_DM_H
#define CIPHER_SHIM_DM_H

#include "petsc_shim.h"

#define SHIM_POOL 8
#define SHIM_MAXLABEL 8

struct _p_Vec {
    double *a;
    int n;
    int local;
    int owns;
    DM dm;
};

struct _p_DMLabel {
    char name[64];
    int npoints;
    PetscInt *values;
    PetscInt defval;
};

struct _p_IS {
    int n;
    PetscInt *idx;
};

struct shim_section {
    int npoints;
    int ndof;
};

struct _p_DM {
    int dim;
    int ncells, nowned, nfaces, nbfaces, ndof;
    PetscInt *cone_off;     /* [ncells+1] */
    PetscInt *cone;         /* face points of each cell */
    PetscInt *support;      /* [2*(nfaces+nbfaces)] */
    double *cellgeom;       /* [ncells] */
    double *centroid;       /* [3*ncells] or NULL */
    const double *ghost;    /* [(ncells-nowned)*ndof] halo values for DMGlobalToLocal */
    struct shim_section lsec, gsec;
    Vec lpool[SHIM_POOL], gpool[SHIM_POOL];
    int lused[SHIM_POOL], gused[SHIM_POOL];
    DMLabel labels[SHIM_MAXLABEL];
    int nlabels;
};

struct _p_TS {
    Vec sol;
    void *ctx;
    double t, dt;
    PetscInt step;
};

Vec shim_vec_wrap(DM dm, double *a, int n, int local);
void shim_vec_free(Vec v);
DMLabel shim_label_new(DM dm, const char *name, int npoints);
extern int shim_verbose;
extern char shim_config_path[PETSC_MAX_PATH_LEN];

#endif
