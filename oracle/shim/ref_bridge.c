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
#include <time.h>
#include "shim_dm.h"
#include "typedef.h"
#include "material.h"
#include "utility.h"
#include "cipher_problem.h"

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
    if (p->gradient_calculation) {
        fprintf(stderr, "ref_bridge: gradient_calculation needs the LSQ matrix of main(); not built\n");
        return 1;
    }

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
    u->nsites = 0;
    u->nnuclei = 0;
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
    for (int i = 0; i < g_dm.nlabels; i++) { free(g_dm.labels[i]->values); free(g_dm.labels[i]); }
    free(g_user.localcells);
    free(g_user.localfaces);
    memset(&g_dm, 0, sizeof(g_dm));
    g_ready = 0;
}
