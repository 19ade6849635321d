/*
 * ref_bridge.c - drives the reference's own RHSFunction and PostStep
 * (src/cipher.c:27-681, 686-1095), compiled unmodified against the PETSc
 * shim, on a problem described by include/cipher_problem.h.
 *
 * Test infrastructure: this is the oracle built from the reference sources
 * (oracle/_ref), used only to check the product and to time the reference
 * on host cores.
 *
 * It fills the reference's AppCtx (src/typedef.h:277-319) the way
 * SetUpConfig would (src/init.c:104-1716) and builds the shim DM from the
 * explicit mesh.  One problem at a time per process: the reference keeps its
 * field sizes and model tables in globals (src/typedef.c, material.c:43-45).
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <math.h>
#include <time.h>
#include "shim_dm.h"
#include "typedef.h"
#include "material.h"
#include "utility.h"
#include "cipher_problem.h"
#include "cipher_b200.h"

extern PetscErrorCode RHSFunction(TS, PetscReal, Vec, Vec, void *);
extern PetscErrorCode PostStep(TS);

#ifndef CIPHER_REF_HAVE_INIT
/* SetUpConfig/SetUpProblem live in src/init.c, which needs libyaml; when
 * init.c is not compiled in, main()'s references resolve here. */
PetscErrorCode SetUpConfig(AppCtx *u) { (void)u; return 1; }
PetscErrorCode SetUpProblem(Vec v, AppCtx *u) { (void)v; (void)u; return 1; }
#else
extern PetscErrorCode SetUpProblem(Vec, AppCtx *);
#endif

static AppCtx g_user;
static struct _p_DM g_dm;
static struct _p_TS g_ts;
static int g_ready = 0;
static int g_sf_rhs = 0;   /* SF_SIZE the reference derives from the config */

/* nucleation tables handed to the next ref_create (ref_set_nuclei) */
static NUCLEUS *g_nuclei = NULL;
static int g_nnuclei = 0, g_nsites = 0;
static PetscInt *g_sitephase = NULL, *g_sitenucleus = NULL;

/* output: a DM of noutputs values per cell and the array VecView copies to */
static struct _p_DM g_dmout;

static void to_tseries(TSeries *d, const cipher_tseries *s)
{
    memset(d, 0, sizeof(*d));
    d->nTser = s->n;
    for (int i = 0; i < s->n && i < 10; i++) { d->exp[i] = s->exp[i]; d->coeff[i] = s->coeff[i]; }
    d->logCoeff = s->logcoeff;
}

static TSeries *tseries_array(const cipher_tseries *s, int n)
{
    TSeries *a = (TSeries *)calloc((size_t)(n > 0 ? n : 1), sizeof(TSeries));
    for (int i = 0; i < n; i++) to_tseries(&a[i], &s[i]);
    return a;
}

static RK *rk_array(const cipher_rk *s, int n)
{
    RK *a = (RK *)calloc((size_t)(n > 0 ? n : 1), sizeof(RK));
    for (int k = 0; k < n; k++) {
        a[k].n = s[k].n;
        a[k].i = (PetscInt *)calloc((size_t)(s[k].n > 0 ? s[k].n : 1), sizeof(PetscInt));
        a[k].enthalpy = (TSeries *)calloc((size_t)(s[k].n > 0 ? s[k].n : 1), sizeof(TSeries));
        for (int r = 0; r < s[k].n; r++) {
            a[k].i[r] = s[k].i[r];
            to_tseries(&a[k].enthalpy[r], &s[k].h[r]);
        }
    }
    return a;
}

static TACTIVATIONPROP *mobility_array(const cipher_mobility *s, int ncp)
{
    TACTIVATIONPROP *a = (TACTIVATIONPROP *)calloc((size_t)ncp, sizeof(TACTIVATIONPROP));
    int nb = ncp * (ncp - 1) / 2;
    for (int c = 0; c < ncp; c++) {
        a[c].m0 = s[c].m0;
        a[c].unary = tseries_array(s[c].unary, ncp);
        a[c].binary = rk_array(s[c].binary, nb);
    }
    return a;
}

static void sources_of(SOURCES *d, const cipher_source *s, int n, int ncp)
{
    d->nsources = n;
    d->sourcename = NULL;
    d->source = (SOURCE *)calloc((size_t)(n > 0 ? n : 1), sizeof(SOURCE));
    for (int i = 0; i < n; i++) {
        d->source[i].source_model = (source_model_t)s[i].model;
        if (s[i].model == CIPHER_SOURCE_SINK) {
            d->source[i].source.sink.rate = (PetscReal *)malloc((size_t)ncp * sizeof(PetscReal));
            d->source[i].source.sink.ceq = (PetscReal *)malloc((size_t)ncp * sizeof(PetscReal));
            memcpy(d->source[i].source.sink.rate, s[i].rate, (size_t)ncp * sizeof(double));
            memcpy(d->source[i].source.sink.ceq, s[i].ceq, (size_t)ncp * sizeof(double));
        } else {
            d->source[i].source.rnd.fluctuation_amplitute = (PetscReal *)malloc((size_t)ncp * sizeof(PetscReal));
            memcpy(d->source[i].source.rnd.fluctuation_amplitute, s[i].amplitude, (size_t)ncp * sizeof(double));
        }
    }
}

static int build_appctx(const cipher_problem *p)
{
    AppCtx *u = &g_user;
    memset(u, 0, sizeof(*u));
    int ncp = p->ncp, ndp = p->ndp, dim = p->dim;
    u->worldrank = 0;
    u->worldsize = 1;
    u->npf = p->npf;
    u->ncp = ncp;
    u->ndp = ndp;
    u->nf = p->nf;
    u->nmat = p->nmat;
    u->nbcs = p->nbcs;
    u->dim = dim;
    u->resolution = (PetscInt *)malloc(3 * sizeof(PetscInt));
    u->size = (PetscReal *)malloc(3 * sizeof(PetscReal));
    for (int d = 0; d < 3; d++) { u->resolution[d] = p->resolution[d]; u->size[d] = p->size[d]; }
    u->gradient_calculation = p->gradient_calculation;

    /* field sizes (src/init.c:1330-1343) */
    MAXSITES = p->maxsites;
    SF_SIZE = MAXSITES * ncp;
    SP_SIZE = MAXSITES * ndp;
    AS_OFFSET = 0;
    AS_SIZE = p->pf_size + 1;
    PF_OFFSET = AS_OFFSET + AS_SIZE;
    PF_SIZE = p->pf_size;
    DP_OFFSET = PF_OFFSET + PF_SIZE;
    DP_SIZE = ndp;
    EX_OFFSET = DP_OFFSET + DP_SIZE;
    EX_SIZE = PF_SIZE * SP_SIZE;
    TM_OFFSET = EX_OFFSET + EX_SIZE;
    TM_SIZE = 1;
    g_sf_rhs = SF_SIZE;

    /* solution parameters */
    u->solparams.nloadcases = p->nloadcases;
    u->solparams.currentloadcase = p->currentloadcase;
    u->solparams.time = (PetscReal *)malloc((size_t)CIPHER_MAXLC * sizeof(PetscReal));
    memcpy(u->solparams.time, p->time, (size_t)CIPHER_MAXLC * sizeof(double));
    if (p->has_temperature_rate) {
        u->solparams.temperature_rate = (PetscReal *)malloc((size_t)CIPHER_MAXLC * sizeof(PetscReal));
        memcpy(u->solparams.temperature_rate, p->temperature_rate, (size_t)CIPHER_MAXLC * sizeof(double));
    } else u->solparams.temperature_rate = NULL;
    u->solparams.timestep = p->timestep0;
    u->solparams.mintimestep = p->mintimestep;
    u->solparams.maxtimestep = p->maxtimestep;
    u->solparams.junctionpenalty = p->junctionpenalty;
    u->solparams.interpolation = (interpolation_t)p->interpolation;
    u->solparams.reltol = p->reltol;
    u->solparams.abstol = p->abstol;
    u->solparams.outputfreq = 0x7fffffff;   /* no VTU output from PostStep */
    strcpy(u->solparams.outfile, "oracle");

    /* materials */
    u->material = (MATERIAL *)calloc((size_t)p->nmat, sizeof(MATERIAL));
    for (int m = 0; m < p->nmat; m++) {
        const cipher_material *s = &p->material[m];
        MATERIAL *d = &u->material[m];
        d->chemfe_model = (chemfe_model_t)s->model;
        d->nsites = s->nsites;
        d->molarvolume = s->molarvolume;
        d->chempot_ex_kineticcoeff = s->chempot_ex_kineticcoeff;
        int ns = s->nsites > 0 ? s->nsites : 1;
        d->c0 = (PetscReal *)calloc((size_t)ns * ncp, sizeof(PetscReal));
        memcpy(d->c0, s->c0, (size_t)ns * ncp * sizeof(double));
        d->stochiometry = (PetscReal *)calloc((size_t)ns, sizeof(PetscReal));
        memcpy(d->stochiometry, s->stoichiometry, (size_t)ns * sizeof(double));
        int c2 = ncp * (ncp - 1) / 2, c3 = ncp * (ncp - 1) * (ncp - 2) / 6;
        switch (s->model) {
        case CIPHER_CHEM_NONE:
            to_tseries(&d->energy.none.ref, &s->ref);
            break;
        case CIPHER_CHEM_QUADRATIC:
            to_tseries(&d->energy.quad.ref, &s->ref);
            d->energy.quad.ceq = tseries_array(s->quad_ceq, ncp);
            d->energy.quad.unary = tseries_array(s->unary, ncp);
            d->energy.quad.binary = tseries_array(s->quad_binary, ncp);
            d->energy.quad.mobilityc = mobility_array(s->mobilityc, ncp);
            break;
        case CIPHER_CHEM_CALPHADDIS:
            to_tseries(&d->energy.calphaddis.ref, &s->ref);
            d->energy.calphaddis.unary = tseries_array(s->unary, ncp);
            d->energy.calphaddis.binary = rk_array(s->binary, c2);
            d->energy.calphaddis.ternary = rk_array(s->ternary, c3);
            d->energy.calphaddis.mobilityc = mobility_array(s->mobilityc, ncp);
            break;
        case CIPHER_CHEM_CALPHAD2SL:
            d->energy.calphad2sl.p = s->p;
            d->energy.calphad2sl.q = s->q;
            d->energy.calphad2sl.unary = tseries_array(s->unary, ncp * ncp);
            d->energy.calphad2sl.binaryp = rk_array(s->binary, c2 * ncp);
            d->energy.calphad2sl.binaryq = rk_array(s->binaryq, c2 * ncp);
            d->energy.calphad2sl.ternaryp = rk_array(s->ternary, c3 * ncp);
            d->energy.calphad2sl.ternaryq = rk_array(s->ternaryq, c3 * ncp);
            d->energy.calphad2sl.mobilityc = mobility_array(s->mobilityc, ncp);
            break;
        default:
            return 1;
        }
        d->thermal.temperature0 = s->temperature0;
        to_tseries(&d->thermal.specific_heat, &s->specific_heat);
        to_tseries(&d->thermal.latent_heat, &s->latent_heat);
        to_tseries(&d->thermal.tconductivity, &s->tconductivity);
        sources_of(&d->sources, s->sources, s->nsources, ncp);
    }

    /* interfaces */
    u->interface = (INTERFACE *)calloc((size_t)p->nf, sizeof(INTERFACE));
    for (int i = 0; i < p->nf; i++) {
        const cipher_interface *s = &p->interface[i];
        INTERFACE *d = &u->interface[i];
        d->ienergy = (IENERGY *)calloc(1, sizeof(IENERGY));
        d->ienergy->e = (TACTIVATIONPROP *)calloc(1, sizeof(TACTIVATIONPROP));
        d->ienergy->e->m0 = s->energy_m0;
        d->ienergy->e->unary = tseries_array(&s->energy_activation, 1);
        d->ienergy->n = s->energy_naniso;
        d->ienergy->dir = (PetscReal *)calloc((size_t)(dim * s->energy_naniso + 1), sizeof(PetscReal));
        d->ienergy->val = (PetscReal *)calloc((size_t)(s->energy_naniso + 1), sizeof(PetscReal));
        memcpy(d->ienergy->dir, s->energy_aniso_dir, (size_t)dim * s->energy_naniso * sizeof(double));
        memcpy(d->ienergy->val, s->energy_aniso_val, (size_t)s->energy_naniso * sizeof(double));
        d->imobility = (IMOBILITY *)calloc(1, sizeof(IMOBILITY));
        d->imobility->m = (TACTIVATIONPROP *)calloc(1, sizeof(TACTIVATIONPROP));
        d->imobility->m->m0 = s->mobility_m0;
        d->imobility->m->unary = tseries_array(&s->mobility_activation, 1);
        d->imobility->n = s->mobility_naniso;
        d->imobility->dir = (PetscReal *)calloc((size_t)(dim * s->mobility_naniso + 1), sizeof(PetscReal));
        d->imobility->val = (PetscReal *)calloc((size_t)(s->mobility_naniso + 1), sizeof(PetscReal));
        memcpy(d->imobility->dir, s->mobility_aniso_dir, (size_t)dim * s->mobility_naniso * sizeof(double));
        memcpy(d->imobility->val, s->mobility_aniso_val, (size_t)s->mobility_naniso * sizeof(double));
        if (s->has_potential) {
            d->potential = (PetscReal *)malloc((size_t)(ndp > 0 ? ndp : 1) * sizeof(PetscReal));
            memcpy(d->potential, s->potential, (size_t)ndp * sizeof(double));
        } else d->potential = NULL;
        if (s->has_mobilityc) {
            d->mobilityc = (PetscReal *)malloc((size_t)ncp * sizeof(PetscReal));
            memcpy(d->mobilityc, s->mobilityc, (size_t)ncp * sizeof(double));
        } else d->mobilityc = NULL;
        d->width = s->width;
        sources_of(&d->isources, s->sources, s->nsources, ncp);
    }
    u->interfacelist = p->interfacelist;
    u->phasematerialmapping = p->phasematerialmapping;

    /* boundary conditions */
    u->bcs = (BOUNDARYCONDITIONS *)calloc((size_t)(p->nbcs > 0 ? p->nbcs : 1), sizeof(BOUNDARYCONDITIONS));
    for (int b = 0; b < p->nbcs; b++) {
        const cipher_bc *s = &p->bcs[b];
        BOUNDARYCONDITIONS *d = &u->bcs[b];
        d->boundaryid = s->boundaryid;
        d->chem_bctype = (boundary_t)s->chem_bctype;
        d->thermal_bctype = (boundary_t)s->thermal_bctype;
        d->chem_bcval = (PetscReal *)calloc((size_t)ncp, sizeof(PetscReal));
        memcpy(d->chem_bcval, s->chem_bcval, (size_t)ncp * sizeof(double));
        d->thermal_bcval = s->thermal_bcval;
        d->chem_bcbool = (char *)calloc((size_t)ncp, 1);
        for (int c = 0; c < ncp; c++) d->chem_bcbool[c] = s->chem_bcbool[c];
    }
    /* nuclei and site mappings (src/init.c:1150-1330) for the reference's
     * NucleationBarrier/NucleationEvent; nsites stays 0 so that PostStep
     * skips its site loop, which needs the distributed site label */
    u->nsites = 0;
    u->nnuclei = g_nnuclei;
    u->nucleus = g_nuclei;
    u->sitephasemapping = g_sitephase;
    u->sitenucleusmapping = g_sitenucleus;
    u->noutputs = 0;
    utility_init(u);
    material_init(u);
    return 0;
}

static int build_dm(const cipher_mesh *m, int ndof)
{
    struct _p_DM *dm = &g_dm;
    memset(dm, 0, sizeof(*dm));
    dm->dim = m->dim;
    dm->ncells = m->ncells;
    dm->nowned = m->nowned;
    dm->nfaces = m->nfaces;
    dm->nbfaces = m->nbfaces;
    dm->ndof = ndof;
    dm->lsec.npoints = m->ncells;
    dm->lsec.ndof = ndof;
    dm->gsec.npoints = m->nowned;
    dm->gsec.ndof = ndof;
    dm->cellgeom = m->cellgeom;
    int nfp = m->nfaces + m->nbfaces;
    dm->support = (PetscInt *)malloc((size_t)(2 * nfp + 2) * sizeof(PetscInt));
    dm->cone_off = (PetscInt *)calloc((size_t)m->ncells + 1, sizeof(PetscInt));
    for (int f = 0; f < m->nfaces; f++) {
        dm->support[2 * f] = m->face_cells[2 * f];
        dm->support[2 * f + 1] = m->face_cells[2 * f + 1];
        dm->cone_off[m->face_cells[2 * f] + 1]++;
        if (m->face_cells[2 * f + 1] != m->face_cells[2 * f]) dm->cone_off[m->face_cells[2 * f + 1] + 1]++;
    }
    for (int b = 0; b < m->nbfaces; b++) {
        dm->support[2 * (m->nfaces + b)] = m->bface_cell[b];
        dm->support[2 * (m->nfaces + b) + 1] = -1;
        dm->cone_off[m->bface_cell[b] + 1]++;
    }
    for (int c = 0; c < m->ncells; c++) dm->cone_off[c + 1] += dm->cone_off[c];
    dm->cone = (PetscInt *)malloc((size_t)(dm->cone_off[m->ncells] + 1) * sizeof(PetscInt));
    int *fill = (int *)calloc((size_t)m->ncells, sizeof(int));
    for (int f = 0; f < m->nfaces; f++) {
        int L = m->face_cells[2 * f], R = m->face_cells[2 * f + 1];
        dm->cone[dm->cone_off[L] + fill[L]++] = m->ncells + f;
        if (R != L) dm->cone[dm->cone_off[R] + fill[R]++] = m->ncells + f;
    }
    for (int b = 0; b < m->nbfaces; b++) {
        int c = m->bface_cell[b];
        dm->cone[dm->cone_off[c] + fill[c]++] = m->ncells + m->nfaces + b;
    }
    free(fill);
    /* boundary label on face points (src/cipher.c:1209-1221) */
    DMLabel bl = shim_label_new(dm, "boundary", m->ncells + nfp);
    for (int b = 0; b < m->nbfaces; b++) bl->values[m->ncells + m->nfaces + b] = m->bface_label[b];
    return 0;
}

/* the least-squares gradient weights main() builds when gradient_calculation
 * is set (src/cipher.c:1232-1282), restated over the shim DM: cell
 * centroids of the uniform grid ((i + 0.5) * size / resolution per axis,
 * from the cell's grid index), the neighbours of each owned cell in its cone
 * order, the reference's Invertmatrix */
static int build_gradient_matrix(const cipher_problem *p, const cipher_mesh *m)
{
    AppCtx *u = &g_user;
    struct _p_DM *dm = &g_dm;
    const int dim = p->dim;
    if (!m->uniform) return 1;
    dm->centroid = (double *)calloc((size_t)3 * m->ncells, sizeof(double));
    if (!dm->centroid) return 1;
    for (int c = 0; c < m->ncells; c++) {
        int64_t g = m->cell_global[c];
        for (int d = 0; d < dim; d++) {
            const int64_t i = g % p->resolution[d];
            g /= p->resolution[d];
            dm->centroid[3 * c + d] = ((double)i + 0.5) * (p->size[d] / p->resolution[d]);
        }
    }
    u->gradient_matrix = (PetscReal *)malloc((size_t)24 * dim * u->nlocalcells * sizeof(PetscReal));
    u->gradient_nleastsq = (PetscInt *)malloc((size_t)u->nlocalcells * sizeof(PetscInt));
    if (!u->gradient_matrix || !u->gradient_nleastsq) return 1;
    for (PetscInt localcell = 0; localcell < u->nlocalcells; ++localcell) {
        const PetscInt cell = u->localcells[localcell];
        PetscReal centroid[3], a_mat[24 * 3], ata_mat[9], atainv_mat[9];
        PetscInt conesize, nsupp;
        const PetscInt *cone, *scells;
        DMPlexComputeCellGeometryFVM(dm, cell, NULL, centroid, NULL);
        DMPlexGetConeSize(dm, cell, &conesize);
        DMPlexGetCone(dm, cell, &cone);
        PetscInt nls = 0;
        for (PetscInt face = 0; face < conesize; face++) {
            DMPlexGetSupportSize(dm, cone[face], &nsupp);
            DMPlexGetSupport(dm, cone[face], &scells);
            for (PetscInt supp = 0; supp < nsupp; supp++) {
                if (scells[supp] != cell && scells[supp] < u->ninteriorcells) {
                    if (nls >= 24) return 1;
                    DMPlexComputeCellGeometryFVM(dm, scells[supp], NULL, &a_mat[nls * dim], NULL);
                    for (int d = 0; d < dim; ++d) a_mat[nls * dim + d] -= centroid[d];
                    nls++;
                }
            }
        }
        u->gradient_nleastsq[localcell] = nls;
        for (int i = 0; i < dim; ++i)
            for (int j = i; j < dim; ++j) {
                PetscReal val = 0.0;
                for (PetscInt k = 0; k < nls; ++k) val += a_mat[k * dim + i] * a_mat[k * dim + j];
                ata_mat[i * dim + j] = val;
                ata_mat[j * dim + i] = val;
            }
        Invertmatrix(atainv_mat, ata_mat, dim);
        PetscReal *gm = &u->gradient_matrix[24 * dim * localcell];
        memset(gm, 0, (size_t)dim * nls * sizeof(PetscReal));
        for (int i = 0; i < dim; ++i)
            for (PetscInt j = 0; j < nls; ++j)
                for (int d = 0; d < dim; ++d) gm[i * nls + j] += atainv_mat[i * dim + d] * a_mat[j * dim + d];
    }
    return 0;
}

int ref_create(const cipher_problem *p, const cipher_mesh *m)
{
    if (g_ready) return 1;
    if (build_appctx(p)) return 2;
    int ndof = AS_SIZE + PF_SIZE + DP_SIZE + EX_SIZE + TM_SIZE;
    if (build_dm(m, ndof)) return 3;
    g_user.da_solution = &g_dm;
    g_user.localcells = (PetscInt *)malloc((size_t)(m->nowned > 0 ? m->nowned : 1) * sizeof(PetscInt));
    for (int c = 0; c < m->nowned; c++) g_user.localcells[c] = c;
    g_user.nlocalcells = m->nowned;
    g_user.ninteriorcells = m->ncells;
    g_user.localfaces = (PetscInt *)malloc((size_t)(m->nfaces > 0 ? m->nfaces : 1) * sizeof(PetscInt));
    for (int f = 0; f < m->nfaces; f++) g_user.localfaces[f] = m->ncells + f;
    g_user.nlocalfaces = m->nfaces;
    g_user.cellgeom = m->cellgeom;
    if (p->gradient_calculation && build_gradient_matrix(p, m)) return 4;
    memset(&g_ts, 0, sizeof(g_ts));
    g_ts.ctx = &g_user;
    g_ready = 1;
    return 0;
}

int ref_ndof(void) { return g_ready ? g_dm.ndof : -1; }

/* ---- calls on a thread with a stack large enough for the RHS's VLAs ---- */

struct call_args {
    int kind;
    double t, dt;
    int step;
    double *X;
    const double *ghost;
    double *F;
    int rc;
    double seconds;
};

static double now_seconds(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void *call_main(void *arg)
{
    struct call_args *a = (struct call_args *)arg;
    g_dm.ghost = a->ghost;
    if (a->kind == 0) {
        Vec X = shim_vec_wrap(&g_dm, a->X, g_dm.nowned * g_dm.ndof, 0);
        Vec F = shim_vec_wrap(&g_dm, a->F, g_dm.nowned * g_dm.ndof, 0);
        SF_SIZE = g_sf_rhs;
        double t0 = now_seconds();
        a->rc = RHSFunction(&g_ts, a->t, X, F, &g_user);
        a->seconds = now_seconds() - t0;
        shim_vec_free(X);
        shim_vec_free(F);
    } else {
        /* With every material `none`, MAXSITES is 0 and the reference's
         * SitepotentialExplicit memsets ncp doubles into a zero-length VLA
         * (src/material.c:642-644).  SF_SIZE only sizes that scratch array in
         * PostStep/SetUpProblem, so it is raised to ncp there; no field
         * offset depends on it. */
        if (SF_SIZE < g_user.ncp) SF_SIZE = g_user.ncp;
        Vec X = shim_vec_wrap(&g_dm, a->X, g_dm.nowned * g_dm.ndof, 0);
        g_ts.sol = X;
        g_ts.t = a->t;
        g_ts.dt = a->dt;
        g_ts.step = a->step;
        double t0 = now_seconds();
        if (a->kind == 1) a->rc = PostStep(&g_ts);
#ifdef CIPHER_REF_HAVE_INIT
        else a->rc = SetUpProblem(X, &g_user);
#else
        else a->rc = 1;
#endif
        a->seconds = now_seconds() - t0;
        a->dt = g_ts.dt;
        g_ts.sol = NULL;
        shim_vec_free(X);
        SF_SIZE = g_sf_rhs;
    }
    return NULL;
}

static int run_big_stack(struct call_args *a)
{
    size_t n = (size_t)g_dm.ncells;
    size_t need = 8 * n * (size_t)(PF_SIZE * (SF_SIZE > g_user.ncp ? SF_SIZE : g_user.ncp) + 2 * g_user.ncp + 2);
    size_t stack = need + ((size_t)64 << 20);
    pthread_attr_t attr;
    pthread_t th;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, stack);
    if (pthread_create(&th, &attr, call_main, a)) { pthread_attr_destroy(&attr); return -1; }
    pthread_join(th, NULL);
    pthread_attr_destroy(&attr);
    return a->rc;
}

/* F (owned cells, AoS) = reference RHSFunction(t, X); ghost = halo cells' values */
int ref_rhs(double t, const double *X, const double *ghost, double *F, double *seconds)
{
    if (!g_ready) return -2;
    struct call_args a = {0};
    a.kind = 0;
    a.t = t;
    a.X = (double *)X;
    a.ghost = ghost;
    a.F = F;
    int rc = run_big_stack(&a);
    if (seconds) *seconds = a.seconds;
    return rc;
}

/* reference PostStep on X (owned cells, AoS) in place; returns the (possibly
 * reset) time step through dt_inout */
int ref_poststep(double *X, double t, double *dt_inout, int step, double *seconds)
{
    if (!g_ready) return -2;
    if (g_dm.ncells != g_dm.nowned) return -3;   /* halo of pruned sets not modelled */
    struct call_args a = {0};
    a.kind = 1;
    a.t = t;
    a.dt = dt_inout ? *dt_inout : 0.0;
    a.step = step;
    a.X = X;
    int rc = run_big_stack(&a);
    if (dt_inout) *dt_inout = a.dt;
    if (seconds) *seconds = a.seconds;
    return rc;
}

/* reference SetUpProblem (src/init.c:1721-1830) into X, phase label from voxel map */
int ref_setup_problem(double *X, const int32_t *cellphase)
{
    if (!g_ready) return -2;
#ifdef CIPHER_REF_HAVE_INIT
    if (g_dm.ncells != g_dm.nowned) return -3;
    DMLabel pl = NULL;
    DMGetLabel(&g_dm, "phase", &pl);
    if (!pl) pl = shim_label_new(&g_dm, "phase", g_dm.ncells + g_dm.nfaces + g_dm.nbfaces);
    for (int c = 0; c < g_dm.ncells; c++) pl->values[c] = cellphase[c];
    memset(X, 0, (size_t)g_dm.nowned * g_dm.ndof * sizeof(double));
    struct call_args a = {0};
    a.kind = 2;
    a.X = X;
    return run_big_stack(&a);
#else
    (void)X; (void)cellphase;
    return -4;
#endif
}

/* release the mesh-side objects so that another problem can be set up; the
 * reference's own model tables (material_init) are process-lifetime */
void ref_destroy(void)
{
    if (!g_ready) return;
    for (int i = 0; i < SHIM_POOL; i++) {
        shim_vec_free(g_dm.lpool[i]);
        shim_vec_free(g_dm.gpool[i]);
    }
    free(g_dm.cone_off);
    free(g_dm.cone);
    free(g_dm.support);
    free(g_dm.centroid);
    free(g_user.gradient_matrix);
    free(g_user.gradient_nleastsq);
    g_user.gradient_matrix = NULL;
    g_user.gradient_nleastsq = NULL;
    for (int i = 0; i < g_dm.nlabels; i++) { free(g_dm.labels[i]->values); free(g_dm.labels[i]); }
    free(g_user.localcells);
    free(g_user.localfaces);
    memset(&g_dm, 0, sizeof(g_dm));
    /* nuclei apply to one problem */
    g_nuclei = NULL;
    g_nnuclei = g_nsites = 0;
    g_sitephase = g_sitenucleus = NULL;
    g_ready = 0;
}

/* ---- nucleation: the reference's per-cell barrier and its events ---- */

/* nuclei (the reference's NUCLEUS, src/typedef.h:105-142, filled as
 * src/init.c reads them) and the site -> phase / nucleus maps; takes effect
 * at the next ref_create */
int ref_set_nuclei(int nsites, const int32_t *sitephase, const int32_t *sitenucleus, int nnuclei,
                   const cipher_nucleus *nz)
{
    if (g_ready) return 1;
    g_nnuclei = nnuclei;
    g_nsites = nsites;
    g_nuclei = (NUCLEUS *)calloc((size_t)(nnuclei > 0 ? nnuclei : 1), sizeof(NUCLEUS));
    g_sitephase = (PetscInt *)calloc((size_t)(nsites > 0 ? nsites : 1), sizeof(PetscInt));
    g_sitenucleus = (PetscInt *)calloc((size_t)(nsites > 0 ? nsites : 1), sizeof(PetscInt));
    for (int s = 0; s < nsites; s++) { g_sitephase[s] = sitephase[s]; g_sitenucleus[s] = sitenucleus[s]; }
    for (int k = 0; k < nnuclei; k++) {
        const cipher_nucleus *a = &nz[k];
        NUCLEUS *d = &g_nuclei[k];
        d->nuc_model = (nucleation_model_t)a->model;
        d->matrixlist = (uint16_t *)calloc((size_t)a->nmatrix + 1, sizeof(uint16_t));
        d->matrixlist[0] = (uint16_t)a->nmatrix;
        for (int i = 0; i < a->nmatrix; i++) d->matrixlist[i + 1] = (uint16_t)a->matrix[i];
        d->activesolutes = (char *)calloc(CIPHER_MAXCP, 1);
        for (int c = 0; c < CIPHER_MAXCP; c++) d->activesolutes[c] = a->active_solutes[c];
        if (a->model == CIPHER_NUC_CONSTANT) {
            d->nucleation.constant.nucleation_rate = a->nucleation_rate;
            d->nucleation.constant.incubationtimemin = a->incubationtimemin;
        } else if (a->model == CIPHER_NUC_CNT) {
            CNT_NUC *c = &d->nucleation.cnt;
            c->gamma = a->gamma; c->shapefactor = a->shapefactor; c->minsize = a->minsize;
            c->atomicvolume = a->atomicvolume; c->lengthscale = a->lengthscale;
            c->incubationtimemin = a->incubationtimemin; c->liquidus = a->liquidus;
        } else if (a->model == CIPHER_NUC_THERMAL) {
            THERMAL_NUC *c = &d->nucleation.thermal;
            c->gamma = a->gamma; c->shapefactor = a->shapefactor; c->minsize = a->minsize;
            c->atomicvolume = a->atomicvolume; c->lengthscale = a->lengthscale;
            c->incubationtimemin = a->incubationtimemin; c->liquidus = a->liquidus;
            c->solvus_temperature_0 = a->solvus_temperature_0;
            c->enthalpy_fusion_0 = a->enthalpy_fusion_0;
            c->solvus_temperature_c = NULL;
            c->enthalpy_fusion_c = NULL;
            if (a->has_solvus_c) {
                c->solvus_temperature_c = (PetscReal *)calloc(CIPHER_MAXCP, sizeof(PetscReal));
                memcpy(c->solvus_temperature_c, a->solvus_temperature_c, CIPHER_MAXCP * sizeof(double));
            }
            if (a->has_enthalpy_c) {
                c->enthalpy_fusion_c = (PetscReal *)calloc(CIPHER_MAXCP, sizeof(PetscReal));
                memcpy(c->enthalpy_fusion_c, a->enthalpy_fusion_c, CIPHER_MAXCP * sizeof(double));
            }
        }
    }
    return 0;
}

struct nuc_args {
    const double *X;
    const int32_t *cellsite;
    int8_t *active;
    double *out;
    int rc;
};

/* the site loop of PostStep (src/cipher.c:733-815) up to the event draw:
 * per active site, over its cells in increasing order, the matrix check
 * (a phase outside the nucleus' matrix retires the site), the reference's
 * EvalInterpolant and NucleationBarrier, volume-weighted sums; then the
 * averages as the root ranks form them */
static void *nuc_main(void *arg)
{
    struct nuc_args *a = (struct nuc_args *)arg;
    AppCtx *u = &g_user;
    const int ndof = g_dm.ndof, ncp = u->ncp;
    if (SF_SIZE < ncp) SF_SIZE = ncp;
    uint16_t slist[AS_SIZE + 1], inter[AS_SIZE + 1], injL[AS_SIZE + 1], injR[AS_SIZE + 1];
    PetscReal interpolant[PF_SIZE + 1], diffusivity[CIPHER_MAXCP], barrier;
    for (int site = 0; site < g_nsites; site++) {
        double *o = &a->out[4 * site];
        o[0] = o[1] = o[2] = o[3] = NAN;
        if (!a->active[site]) continue;
        const NUCLEUS *nz = &u->nucleus[u->sitenucleusmapping[site]];
        double gv = 0.0, vol = 0.0, tsum = 0.0, dsum[CIPHER_MAXCP] = {0};
        int retire = 0;
        for (int cell = 0; cell < g_dm.nowned; cell++) {
            if (a->cellsite[cell] != site) continue;
            double *off = (double *)&a->X[(size_t)cell * ndof];
            F2IFUNC(slist, &off[AS_OFFSET]);
            SetIntersection(inter, injL, injR, slist, nz->matrixlist);
            if (inter[0] != slist[0]) { retire = 1; break; }
            EvalInterpolant(interpolant, &off[PF_OFFSET], slist[0]);
            NucleationBarrier(&barrier, diffusivity, &off[DP_OFFSET], &off[EX_OFFSET], off[TM_OFFSET], interpolant,
                              (uint16_t)site, slist, u);
            const double cv = FastPow(u->cellgeom[cell], u->dim);
            vol += cv;
            tsum += cv * off[TM_OFFSET];
            gv += cv * barrier;
            for (int c = 0; c < ncp; c++) dsum[c] += cv * diffusivity[c];
        }
        if (retire) { a->active[site] = 0; continue; }
        double d = LARGE;
        for (int c = 0; c < ncp; c++)
            if (nz->activesolutes[c]) d = d < dsum[c] ? d : dsum[c];
        o[0] = gv / vol;
        o[1] = d / vol;
        o[2] = tsum / vol;
        o[3] = vol;
    }
    SF_SIZE = g_sf_rhs;
    a->rc = 0;
    return NULL;
}

/* per-site (barrier, diffusivity, temperature, volume) of state X (owned
 * cells, AoS) into out[4*nsites] (NaN for sites not evaluated); active[] is
 * updated for retired sites.  cellsite[cell] = the cell's site or -1 */
int ref_nucleation_sites(const double *X, const int32_t *cellsite, int8_t *active, double *out)
{
    if (!g_ready) return -2;
    struct nuc_args a = {X, cellsite, active, out, -1};
    pthread_attr_t attr;
    pthread_t th;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, (size_t)64 << 20);
    if (pthread_create(&th, &attr, nuc_main, &a)) { pthread_attr_destroy(&attr); return -1; }
    pthread_join(th, NULL);
    pthread_attr_destroy(&attr);
    return a.rc;
}

/* the reference's NucleationEvent for `site` with the C library's generator
 * seeded by `seed`; *draw = the first number that generator gives
 * (rand()/RAND_MAX, the reference's draw), so that a caller can replay the
 * decision with its own probability */
int ref_nucleation_event(int site, double t, double dt, double temperature, double volume, double gv,
                         double diffusivity, unsigned seed, double *draw)
{
    if (!g_ready || site < 0 || site >= g_nsites) return -2;
    srand(seed);
    *draw = rand() / (double)RAND_MAX;
    srand(seed);
    return NucleationEvent(t, dt, temperature, volume, gv, diffusivity, site, &g_user);
}

/* ---- output: the reference's output step (src/cipher.c:976-1093) ---- */

double *shim_capture = NULL;       /* VecView copies its vector here */
int shim_capture_n = 0;

/* reference PostStep on X (owned cells, AoS) in place with output at this
 * step: out[cell*noutputs + o] = field `names[o]` of the post-step state, as
 * the reference writes it to its .vtu file */
int ref_output_fields(double *X, double t, int step, int noutputs, const char *const *names,
                      const char *const *components, double *out)
{
    if (!g_ready) return -2;
    if (g_dm.ncells != g_dm.nowned) return -3;
    struct _p_DM *d = &g_dmout;
    memset(d, 0, sizeof(*d));
    d->dim = g_dm.dim;
    d->ncells = g_dm.ncells;
    d->nowned = g_dm.nowned;
    d->ndof = noutputs;
    d->lsec.npoints = g_dm.ncells;
    d->lsec.ndof = noutputs;
    d->gsec.npoints = g_dm.nowned;
    d->gsec.ndof = noutputs;
    d->cellgeom = g_dm.cellgeom;
    g_user.da_output = d;
    g_user.noutputs = noutputs;
    g_user.outputname = (char **)names;
    g_user.componentname = (char **)components;
    g_user.solparams.outputfreq = 1;
    shim_capture = out;
    shim_capture_n = g_dm.nowned * noutputs;
    struct call_args a = {0};
    a.kind = 1;
    a.t = t;
    a.step = step;
    a.X = X;
    int rc = run_big_stack(&a);
    shim_capture = NULL;
    shim_capture_n = 0;
    g_user.solparams.outputfreq = 0x7fffffff;
    g_user.noutputs = 0;
    g_user.outputname = NULL;
    g_user.componentname = NULL;
    g_user.da_output = NULL;
    for (int i = 0; i < SHIM_POOL; i++) shim_vec_free(d->gpool[i]);
    memset(d, 0, sizeof(*d));
    return rc;
}

/* ---- configuration: the reference's SetUpConfig on replayed YAML events ---- */

#ifdef CIPHER_REF_HAVE_INIT
#include "yaml.h"

extern PetscErrorCode SetUpConfig(AppCtx *);

static int g_nev = 0;
static yaml_event_type_t *g_evtype = NULL;
static unsigned char **g_evval = NULL;
static AppCtx g_cfg;
static int g_cfg_ready = 0;

int yaml_parser_initialize(yaml_parser_t *parser) { parser->pos = 0; return 1; }
void yaml_parser_set_input_string(yaml_parser_t *parser, const unsigned char *input, size_t size)
{
    (void)input; (void)size;
    parser->pos = 0;
}
int yaml_parser_parse(yaml_parser_t *parser, yaml_event_t *event)
{
    memset(event, 0, sizeof(*event));
    if (parser->pos >= g_nev) { event->type = YAML_NO_EVENT; return 0; }
    event->type = g_evtype[parser->pos];
    event->data.scalar.value = g_evval[parser->pos];
    event->data.scalar.length = g_evval[parser->pos] ? strlen((char *)g_evval[parser->pos]) : 0;
    parser->pos++;
    return 1;
}
void yaml_event_delete(yaml_event_t *event) { (void)event; }
void yaml_parser_delete(yaml_parser_t *parser) { (void)parser; }

/* the event stream of the configuration file (types as yaml_event_type_t;
 * values[i] the scalar text of scalar events, else NULL) */
int ref_config_events(int n, const int *types, const char *const *values)
{
    g_evtype = (yaml_event_type_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(yaml_event_type_t));
    g_evval = (unsigned char **)calloc((size_t)(n > 0 ? n : 1), sizeof(unsigned char *));
    if (!g_evtype || !g_evval) return -1;
    for (int i = 0; i < n; i++) {
        g_evtype[i] = (yaml_event_type_t)types[i];
        g_evval[i] = values[i] ? (unsigned char *)strdup(values[i]) : NULL;
    }
    g_nev = n;
    return 0;
}

/* SetUpConfig (src/init.c:104-1716) on the file at `path`, reading the
 * events given to ref_config_events; the reference asserts on a bad file
 * (the process aborts) */
int ref_config_load(const char *path)
{
    memset(&g_cfg, 0, sizeof(g_cfg));
    g_cfg.worldrank = 0;
    g_cfg.worldsize = 1;
    strncpy(shim_config_path, path, PETSC_MAX_PATH_LEN - 1);
    const int rc = SetUpConfig(&g_cfg);
    g_cfg_ready = rc == 0;
    return rc;
}

static void tser_out(cipher_tseries *d, const TSeries *s)
{
    memset(d, 0, sizeof(*d));
    d->n = s->nTser;
    for (int i = 0; i < s->nTser && i < CIPHER_MAXTSER; i++) { d->exp[i] = s->exp[i]; d->coeff[i] = s->coeff[i]; }
    d->logcoeff = s->logCoeff;
}

static void rk_out(cipher_rk *d, const RK *s, int with_index)
{
    memset(d, 0, sizeof(*d));
    d->n = s->n;
    for (int k = 0; k < s->n && k < CIPHER_MAXRK; k++) {
        tser_out(&d->h[k], &s->enthalpy[k]);
        if (with_index) d->i[k] = s->i[k];
    }
}

static void mob_out(cipher_mobility *d, const TACTIVATIONPROP *s, int ncp)
{
    memset(d, 0, sizeof(*d));
    d->m0 = s->m0;
    for (int j = 0; j < ncp; j++) tser_out(&d->unary[j], &s->unary[j]);
    for (int b = 0; b < ncp * (ncp - 1) / 2; b++) rk_out(&d->binary[b], &s->binary[b], 0);
}

static void src_out(int32_t *n, cipher_source *d, const SOURCES *s, int ncp)
{
    *n = s->nsources;
    for (int k = 0; k < s->nsources && k < CIPHER_MAXSRC; k++) {
        memset(&d[k], 0, sizeof(d[k]));
        d[k].model = s->source[k].source_model;
        for (int c = 0; c < ncp; c++) {
            if (d[k].model == CIPHER_SOURCE_SINK) {
                d[k].rate[c] = s->source[k].source.sink.rate[c];
                d[k].ceq[c] = s->source[k].source.sink.ceq[c];
            } else {
                d[k].amplitude[c] = s->source[k].source.rnd.fluctuation_amplitute[c];
            }
        }
    }
}

/* the parsed AppCtx as this project's problem tables (allocated here):
 * info[0..13] = nsites, nnuclei, noutputs, ncp, outputfreq, randomseed,
 * initrefine, initcoarsen, maxnrefine, minnrefine, amrinterval,
 * initblocksize[3] */
int ref_config_export(cipher_problem *p, int64_t *info)
{
    if (!g_cfg_ready) return -2;
    const AppCtx *u = &g_cfg;
    const int ncp = u->ncp, ndp = u->ndp, dim = u->dim, npf = u->npf;
    memset(p, 0, sizeof(*p));
    p->dim = dim;
    p->npf = npf;
    p->ncp = ncp;
    p->ndp = ndp;
    p->nmat = u->nmat;
    p->nf = u->nf;
    p->nbcs = u->nbcs;
    p->pf_size = PF_SIZE;
    p->maxsites = MAXSITES;
    p->interpolation = u->solparams.interpolation;
    p->gradient_calculation = u->gradient_calculation;
    p->junctionpenalty = u->solparams.junctionpenalty;
    p->nloadcases = u->solparams.nloadcases;
    p->currentloadcase = 0;
    for (int i = 0; i < u->solparams.nloadcases && i < CIPHER_MAXLC; i++) p->time[i] = u->solparams.time[i];
    p->has_temperature_rate = u->solparams.temperature_rate != NULL;
    for (int i = 0; p->has_temperature_rate && i < u->solparams.nloadcases && i < CIPHER_MAXLC; i++)
        p->temperature_rate[i] = u->solparams.temperature_rate[i];
    p->timestep0 = u->solparams.timestep;
    p->mintimestep = u->solparams.mintimestep;
    p->maxtimestep = u->solparams.maxtimestep;
    p->reltol = u->solparams.reltol;
    p->abstol = u->solparams.abstol;
    int64_t total = 1;
    for (int d = 0; d < 3; d++) {
        p->resolution[d] = d < dim ? u->resolution[d] : 1;
        p->size[d] = d < dim ? u->size[d] : 1.0;
        total *= p->resolution[d];
    }
    p->material = (cipher_material *)calloc((size_t)u->nmat, sizeof(cipher_material));
    p->interface = (cipher_interface *)calloc((size_t)u->nf, sizeof(cipher_interface));
    p->interfacelist = (int32_t *)calloc((size_t)npf * npf, sizeof(int32_t));
    p->phasematerialmapping = (int32_t *)calloc((size_t)npf, sizeof(int32_t));
    p->voxelphase = (int32_t *)calloc((size_t)total, sizeof(int32_t));
    if (!p->material || !p->interface || !p->interfacelist || !p->phasematerialmapping || !p->voxelphase) return -1;
    for (int m = 0; m < u->nmat; m++) {
        const MATERIAL *s = &u->material[m];
        cipher_material *d = &p->material[m];
        d->model = s->chemfe_model;
        d->nsites = s->nsites;
        d->molarvolume = s->molarvolume;
        d->chempot_ex_kineticcoeff = s->chempot_ex_kineticcoeff;
        if (s->chemfe_model != NONE_CHEMENERGY) {
            for (int i = 0; i < s->nsites * ncp; i++) d->c0[i] = s->c0[i];
            for (int i = 0; i < s->nsites; i++) d->stoichiometry[i] = s->stochiometry[i];
        }
        const int c2 = ncp * (ncp - 1) / 2, c3 = ncp * (ncp - 1) * (ncp - 2) / 6;
        switch (s->chemfe_model) {
        case NONE_CHEMENERGY:
            tser_out(&d->ref, &s->energy.none.ref);
            break;
        case QUADRATIC_CHEMENERGY:
            tser_out(&d->ref, &s->energy.quad.ref);
            for (int c = 0; c < ncp; c++) {
                tser_out(&d->quad_ceq[c], &s->energy.quad.ceq[c]);
                tser_out(&d->unary[c], &s->energy.quad.unary[c]);
                tser_out(&d->quad_binary[c], &s->energy.quad.binary[c]);
                mob_out(&d->mobilityc[c], &s->energy.quad.mobilityc[c], ncp);
            }
            break;
        case CALPHADDIS_CHEMENERGY:
            tser_out(&d->ref, &s->energy.calphaddis.ref);
            for (int c = 0; c < ncp; c++) {
                tser_out(&d->unary[c], &s->energy.calphaddis.unary[c]);
                mob_out(&d->mobilityc[c], &s->energy.calphaddis.mobilityc[c], ncp);
            }
            for (int b = 0; b < c2; b++) rk_out(&d->binary[b], &s->energy.calphaddis.binary[b], 0);
            for (int t = 0; t < c3; t++) rk_out(&d->ternary[t], &s->energy.calphaddis.ternary[t], 1);
            break;
        case CALPHAD2SL_CHEMENERGY:
            d->p = s->energy.calphad2sl.p;
            d->q = s->energy.calphad2sl.q;
            for (int c = 0; c < ncp * ncp; c++) tser_out(&d->unary[c], &s->energy.calphad2sl.unary[c]);
            for (int c = 0; c < ncp; c++) mob_out(&d->mobilityc[c], &s->energy.calphad2sl.mobilityc[c], ncp);
            for (int b = 0; b < c2 * ncp; b++) {
                rk_out(&d->binary[b], &s->energy.calphad2sl.binaryp[b], 0);
                rk_out(&d->binaryq[b], &s->energy.calphad2sl.binaryq[b], 0);
            }
            for (int t = 0; t < c3 * ncp; t++) {
                rk_out(&d->ternary[t], &s->energy.calphad2sl.ternaryp[t], 0);
                rk_out(&d->ternaryq[t], &s->energy.calphad2sl.ternaryq[t], 0);
            }
            break;
        }
        d->temperature0 = s->thermal.temperature0;
        tser_out(&d->specific_heat, &s->thermal.specific_heat);
        tser_out(&d->latent_heat, &s->thermal.latent_heat);
        tser_out(&d->tconductivity, &s->thermal.tconductivity);
        src_out(&d->nsources, d->sources, &s->sources, ncp);
    }
    for (int i = 0; i < u->nf; i++) {
        const INTERFACE *s = &u->interface[i];
        cipher_interface *d = &p->interface[i];
        d->width = s->width;
        d->energy_m0 = s->ienergy->e->m0;
        tser_out(&d->energy_activation, &s->ienergy->e->unary[0]);
        d->energy_naniso = s->ienergy->n;
        for (int k = 0; k < s->ienergy->n; k++) {
            d->energy_aniso_val[k] = s->ienergy->val[k];
            for (int a = 0; a < dim; a++) d->energy_aniso_dir[k * dim + a] = s->ienergy->dir ? s->ienergy->dir[k * dim + a] : 0.0;
        }
        d->mobility_m0 = s->imobility->m->m0;
        tser_out(&d->mobility_activation, &s->imobility->m->unary[0]);
        d->mobility_naniso = s->imobility->n;
        for (int k = 0; k < s->imobility->n; k++) {
            d->mobility_aniso_val[k] = s->imobility->val[k];
            for (int a = 0; a < dim; a++) d->mobility_aniso_dir[k * dim + a] = s->imobility->dir ? s->imobility->dir[k * dim + a] : 0.0;
        }
        d->has_potential = s->potential != NULL;
        for (int c = 0; d->has_potential && c < ndp; c++) d->potential[c] = s->potential[c];
        d->has_mobilityc = s->mobilityc != NULL;
        for (int c = 0; d->has_mobilityc && c < ncp; c++) d->mobilityc[c] = s->mobilityc[c];
        src_out(&d->nsources, d->sources, &s->isources, ncp);
    }
    for (int b = 0; b < u->nbcs && b < CIPHER_MAXBC; b++) {
        const BOUNDARYCONDITIONS *s = &u->bcs[b];
        cipher_bc *d = &p->bcs[b];
        d->boundaryid = s->boundaryid;
        d->chem_bctype = s->chem_bctype;
        d->thermal_bctype = s->thermal_bctype;
        if (s->chem_bctype != NONE_BC)
            for (int c = 0; c < ncp; c++) { d->chem_bcval[c] = s->chem_bcval[c]; d->chem_bcbool[c] = s->chem_bcbool[c]; }
        if (s->thermal_bctype != NONE_BC) d->thermal_bcval = s->thermal_bcval;
    }
    /* the interface table is filled above the diagonal (src/init.c:1501) */
    for (int a = 0; a < npf; a++)
        for (int b = a + 1; b < npf; b++) {
            p->interfacelist[a * npf + b] = (int32_t)u->interfacelist[a * npf + b];
            p->interfacelist[b * npf + a] = (int32_t)u->interfacelist[a * npf + b];
        }
    for (int i = 0; i < npf; i++) p->phasematerialmapping[i] = (int32_t)u->phasematerialmapping[i];
    for (int64_t i = 0; i < total; i++) p->voxelphase[i] = (int32_t)u->voxelphasemapping[i];
    const int64_t v[14] = {u->nsites, u->nnuclei, u->noutputs, ncp, u->solparams.outputfreq,
                           u->solparams.randomseed, u->amrparams.initrefine, u->amrparams.initcoarsen,
                           u->amrparams.maxnrefine, u->amrparams.minnrefine, u->amrparams.amrinterval,
                           dim > 0 ? u->amrparams.initblocksize[0] : 1, dim > 1 ? u->amrparams.initblocksize[1] : 1,
                           dim > 2 ? u->amrparams.initblocksize[2] : 1};
    memcpy(info, v, sizeof(v));
    return 0;
}

/* sites and nuclei of the parsed configuration: voxelsite[total] (the site
 * whose label stratum holds the voxel, -1 for none: label = mapped value - 1,
 * site s = label s+1, src/cipher.c:1308 and 736), sitephase[nsites],
 * sitenucleus[nsites], nuclei[nnuclei] with the matrix list as written */
int ref_config_sites(int32_t *voxelsite, int32_t *sitephase, int32_t *sitenucleus, cipher_nucleus *nuclei)
{
    if (!g_cfg_ready) return -2;
    const AppCtx *u = &g_cfg;
    int64_t total = 1;
    for (int d = 0; d < u->dim; d++) total *= u->resolution[d];
    for (int64_t i = 0; u->nsites && i < total; i++) {
        const PetscInt s = u->voxelsitemapping[i] - 1;
        voxelsite[i] = (s >= 0 && s < u->nsites) ? (int32_t)s : -1;
    }
    for (int s = 0; s < u->nsites; s++) {
        sitephase[s] = (int32_t)u->sitephasemapping[s];
        sitenucleus[s] = (int32_t)u->sitenucleusmapping[s];
    }
    for (int k = 0; k < u->nnuclei; k++) {
        const NUCLEUS *s = &u->nucleus[k];
        cipher_nucleus *d = &nuclei[k];
        memset(d, 0, sizeof(*d));
        d->model = s->nuc_model;
        d->nmatrix = s->matrixlist[0];
        for (int i = 0; i < d->nmatrix && i < 16; i++) d->matrix[i] = s->matrixlist[i + 1];
        for (int c = 0; c < u->ncp; c++) d->active_solutes[c] = s->activesolutes[c];
        if (s->nuc_model == CNT_NUCLEATION) {
            const CNT_NUC *c = &s->nucleation.cnt;
            d->gamma = c->gamma; d->shapefactor = c->shapefactor; d->minsize = c->minsize;
            d->atomicvolume = c->atomicvolume; d->lengthscale = c->lengthscale;
            d->incubationtimemin = c->incubationtimemin; d->liquidus = c->liquidus;
        } else if (s->nuc_model == CONST_NUCLEATION) {
            d->nucleation_rate = s->nucleation.constant.nucleation_rate;
            d->incubationtimemin = s->nucleation.constant.incubationtimemin;
        } else if (s->nuc_model == THERMAL_NUCLEATION) {
            const THERMAL_NUC *c = &s->nucleation.thermal;
            d->gamma = c->gamma; d->shapefactor = c->shapefactor; d->minsize = c->minsize;
            d->atomicvolume = c->atomicvolume; d->lengthscale = c->lengthscale;
            d->incubationtimemin = c->incubationtimemin; d->liquidus = c->liquidus;
            d->solvus_temperature_0 = c->solvus_temperature_0;
            d->enthalpy_fusion_0 = c->enthalpy_fusion_0;
            d->has_solvus_c = c->solvus_temperature_c != NULL;
            d->has_enthalpy_c = c->enthalpy_fusion_c != NULL;
            for (int i = 0; i < u->ncp; i++) {
                if (d->has_solvus_c) d->solvus_temperature_c[i] = c->solvus_temperature_c[i];
                if (d->has_enthalpy_c) d->enthalpy_fusion_c[i] = c->enthalpy_fusion_c[i];
            }
        }
    }
    return 0;
}

/* names of the parsed configuration: kind 0 component, 1 output, 2 outfile,
 * 3 petscoptions (with the brick options the reference appends) */
int ref_config_string(int kind, int index, char *buf, int len)
{
    if (!g_cfg_ready || len < 1) return -2;
    const char *s = NULL;
    if (kind == 0 && index >= 0 && index < g_cfg.ncp) s = g_cfg.componentname[index];
    else if (kind == 1 && index >= 0 && index < g_cfg.noutputs) s = g_cfg.outputname[index];
    else if (kind == 2) s = g_cfg.solparams.outfile;
    else if (kind == 3) s = g_cfg.solparams.petscoptions;
    if (!s) return -1;
    snprintf(buf, (size_t)len, "%s", s);
    return 0;
}
#endif
