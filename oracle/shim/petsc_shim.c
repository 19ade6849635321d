/*
 * petsc_shim.c - explicit-mesh implementation of the PETSc calls made by
 * CIPHER's RHSFunction / PostStep / SetUpProblem (src/cipher.c:27-1095,
 * src/init.c:1721-1830).  Test infrastructure for the CPU oracle.
 *
 * Semantics reproduced (the ones the reference relies on):
 *   - cells are points [0, ncells): owned first, then ghosts;
 *   - a cell's cone is its faces, a face's support is [L, R] (interior)
 *     or [cell] (boundary);
 *   - DMPlexPointLocalRef addresses any cell of a local vector,
 *     DMPlexPointGlobalRef only owned cells of a global vector;
 *   - DMGlobalToLocal copies owned values and fills ghosts from the halo
 *     buffer the caller registered (what the MPI halo exchange delivers).
 */
#include <stdarg.h>
#include "shim_dm.h"

static int shim_unsupported(const char *what)
{
    fprintf(stderr, "petsc shim: %s is not supported\n", what);
    return 1;
}

/* ---------------- MPI ---------------- */
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)n; (void)t; (void)op; (void)c;
    if (in != MPI_IN_PLACE) return shim_unsupported("MPI_Allreduce (not in place)");
    (void)out;
    return 0;
}

/* ---------------- init / printing ---------------- */
PetscErrorCode PetscInitialize(int *a, char ***b, const char *c, const char *d) { (void)a; (void)b; (void)c; (void)d; return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }
int shim_verbose = 0;
PetscErrorCode PetscPrintf(MPI_Comm c, const char *fmt, ...)
{
    (void)c;
    if (!shim_verbose) return 0;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    return 0;
}
PetscErrorCode PetscOptionsInsertString(void *o, const char *s) { (void)o; (void)s; return 0; }
char shim_config_path[PETSC_MAX_PATH_LEN] = "";
PetscErrorCode PetscOptionsGetString(void *o, const char *pre, const char *name, char *val, size_t len, PetscBool *set)
{
    (void)o; (void)pre;
    if (!strcmp(name, "--config") && shim_config_path[0]) {
        strncpy(val, shim_config_path, len - 1);
        val[len - 1] = 0;
        if (set) *set = PETSC_TRUE;
    } else if (set) *set = PETSC_FALSE;
    return 0;
}
PetscErrorCode PetscObjectSetName(PetscObject o, const char *n) { (void)o; (void)n; return 0; }
MPI_Comm PetscObjectComm(PetscObject o) { (void)o; return PETSC_COMM_WORLD; }

/* ---------------- Vec ---------------- */
Vec shim_vec_wrap(DM dm, double *a, int n, int local)
{
    Vec v = (Vec)calloc(1, sizeof(struct _p_Vec));
    v->a = a; v->n = n; v->local = local; v->dm = dm; v->owns = 0;
    return v;
}
static Vec vec_new(DM dm, int n, int local)
{
    Vec v = (Vec)calloc(1, sizeof(struct _p_Vec));
    v->a = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    v->n = n; v->local = local; v->dm = dm; v->owns = 1;
    return v;
}
void shim_vec_free(Vec v)
{
    if (!v) return;
    if (v->owns) free(v->a);
    free(v);
}
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a) { (void)v; *a = NULL; return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a) { (void)v; *a = NULL; return 0; }
PetscErrorCode VecZeroEntries(Vec v) { memset(v->a, 0, (size_t)v->n * sizeof(double)); return 0; }
PetscErrorCode VecCopy(Vec x, Vec y)
{
    if (x->n != y->n) return shim_unsupported("VecCopy of different sizes");
    memcpy(y->a, x->a, (size_t)x->n * sizeof(double));
    return 0;
}
PetscErrorCode VecDestroy(Vec *v) { shim_vec_free(*v); *v = NULL; return 0; }
PetscErrorCode VecGetDM(Vec v, DM *dm) { *dm = v->dm; return 0; }
/* the output step's VecView: the bridge collects the vector (no file is
 * written); any other VecView is not modelled */
extern double *shim_capture;
extern int shim_capture_n;
PetscErrorCode VecView(Vec v, PetscViewer w)
{
    (void)w;
    if (!shim_capture || v->n != shim_capture_n) return shim_unsupported("VecView");
    memcpy(shim_capture, v->a, (size_t)v->n * sizeof(double));
    return 0;
}

/* ---------------- DM: vectors ---------------- */
static Vec pool_get(DM dm, int local)
{
    Vec *pool = local ? dm->lpool : dm->gpool;
    int *used = local ? dm->lused : dm->gused;
    for (int i = 0; i < SHIM_POOL; i++) {
        if (!pool[i]) pool[i] = vec_new(dm, (local ? dm->ncells : dm->nowned) * dm->ndof, local);
        if (!used[i]) { used[i] = 1; return pool[i]; }
    }
    return NULL;
}
static void pool_put(DM dm, Vec v)
{
    for (int i = 0; i < SHIM_POOL; i++) {
        if (dm->lpool[i] == v) { dm->lused[i] = 0; return; }
        if (dm->gpool[i] == v) { dm->gused[i] = 0; return; }
    }
}
PetscErrorCode DMCreateGlobalVector(DM dm, Vec *v) { *v = vec_new(dm, dm->nowned * dm->ndof, 0); return 0; }
PetscErrorCode DMGetLocalVector(DM dm, Vec *v) { *v = pool_get(dm, 1); return *v ? 0 : shim_unsupported("local vector pool"); }
PetscErrorCode DMRestoreLocalVector(DM dm, Vec *v) { pool_put(dm, *v); *v = NULL; return 0; }
PetscErrorCode DMGetGlobalVector(DM dm, Vec *v) { *v = pool_get(dm, 0); return *v ? 0 : shim_unsupported("global vector pool"); }
PetscErrorCode DMRestoreGlobalVector(DM dm, Vec *v) { pool_put(dm, *v); *v = NULL; return 0; }
PetscErrorCode DMGlobalToLocalBegin(DM dm, Vec g, InsertMode m, Vec l)
{
    (void)m;
    if (g->local || !l->local) return shim_unsupported("DMGlobalToLocal direction");
    size_t own = (size_t)dm->nowned * dm->ndof;
    memcpy(l->a, g->a, own * sizeof(double));
    size_t nghost = (size_t)(dm->ncells - dm->nowned) * dm->ndof;
    if (nghost) {
        if (!dm->ghost) return shim_unsupported("ghost values not registered");
        memcpy(l->a + own, dm->ghost, nghost * sizeof(double));
    }
    return 0;
}
PetscErrorCode DMGlobalToLocalEnd(DM dm, Vec g, InsertMode m, Vec l) { (void)dm; (void)g; (void)m; (void)l; return 0; }

/* ---------------- DM: topology ---------------- */
PetscErrorCode DMPlexGetHeightStratum(DM dm, PetscInt h, PetscInt *s, PetscInt *e)
{
    if (h == 0) { *s = 0; *e = dm->ncells; }
    else if (h == 1) { *s = dm->ncells; *e = dm->ncells + dm->nfaces + dm->nbfaces; }
    else { *s = *e = 0; }
    return 0;
}
PetscErrorCode DMPlexGetConeSize(DM dm, PetscInt p, PetscInt *n)
{
    if (p < 0 || p >= dm->ncells) { *n = 0; return 0; }
    *n = dm->cone_off[p + 1] - dm->cone_off[p];
    return 0;
}
PetscErrorCode DMPlexGetCone(DM dm, PetscInt p, const PetscInt **c)
{
    *c = (p >= 0 && p < dm->ncells) ? &dm->cone[dm->cone_off[p]] : NULL;
    return 0;
}
PetscErrorCode DMPlexGetSupportSize(DM dm, PetscInt p, PetscInt *n)
{
    int f = p - dm->ncells;
    if (f < 0) *n = 0;
    else if (f < dm->nfaces) *n = 2;
    else if (f < dm->nfaces + dm->nbfaces) *n = 1;
    else *n = 0;
    return 0;
}
PetscErrorCode DMPlexGetSupport(DM dm, PetscInt p, const PetscInt **s)
{
    int f = p - dm->ncells;
    if (f < 0 || f >= dm->nfaces + dm->nbfaces) { *s = NULL; return 0; }
    *s = &dm->support[2 * f];
    return 0;
}
PetscErrorCode DMPlexGetTreeChildren(DM dm, PetscInt p, PetscInt *n, const PetscInt **c)
{
    (void)dm; (void)p;
    if (n) *n = 0;
    if (c) *c = NULL;
    return 0;
}
PetscErrorCode DMPlexPointLocalRef(DM dm, PetscInt p, PetscScalar *a, void *ptr)
{
    if (p < 0 || p >= dm->ncells) { *(PetscScalar **)ptr = NULL; return 1; }
    *(PetscScalar **)ptr = a + (size_t)p * dm->ndof;
    return 0;
}
PetscErrorCode DMPlexPointGlobalRef(DM dm, PetscInt p, PetscScalar *a, void *ptr)
{
    if (p < 0 || p >= dm->nowned) { *(PetscScalar **)ptr = NULL; return 1; }
    *(PetscScalar **)ptr = a + (size_t)p * dm->ndof;
    return 0;
}
PetscErrorCode DMPlexPointLocalRead(DM dm, PetscInt p, const PetscScalar *a, void *ptr)
{
    if (p < 0 || p >= dm->ncells) { *(const PetscScalar **)ptr = NULL; return 1; }
    *(const PetscScalar **)ptr = a + (size_t)p * dm->ndof;
    return 0;
}
PetscErrorCode DMPlexComputeCellGeometryFVM(DM dm, PetscInt p, PetscReal *vol, PetscReal *cen, PetscReal *nrm)
{
    (void)nrm;
    if (p < 0 || p >= dm->ncells) return shim_unsupported("geometry of a non-cell point");
    if (vol) { double v = 1.0; for (int d = 0; d < dm->dim; d++) v *= dm->cellgeom[p]; *vol = v; }
    if (cen) for (int d = 0; d < dm->dim; d++) cen[d] = dm->centroid ? dm->centroid[3 * p + d] : 0.0;
    return 0;
}
PetscErrorCode DMPlexGetDataFVM(DM dm, void *fv, Vec *cg, Vec *fg, DM *gdm) { (void)dm; (void)fv; (void)cg; (void)fg; (void)gdm; return shim_unsupported("DMPlexGetDataFVM"); }

/* ---------------- sections ---------------- */
PetscErrorCode DMGetSection(DM dm, PetscSection *s) { *s = (PetscSection)&dm->lsec; return 0; }
PetscErrorCode DMGetGlobalSection(DM dm, PetscSection *s) { *s = (PetscSection)&dm->gsec; return 0; }
PetscErrorCode PetscSectionGetDof(PetscSection s, PetscInt p, PetscInt *n)
{
    struct shim_section *sec = (struct shim_section *)s;
    *n = (p >= 0 && p < sec->npoints) ? sec->ndof : 0;
    return 0;
}

/* ---------------- labels ---------------- */
static DMLabel find_label(DM dm, const char *name)
{
    for (int i = 0; i < dm->nlabels; i++)
        if (!strcmp(dm->labels[i]->name, name)) return dm->labels[i];
    return NULL;
}
DMLabel shim_label_new(DM dm, const char *name, int npoints)
{
    DMLabel l = (DMLabel)calloc(1, sizeof(struct _p_DMLabel));
    strncpy(l->name, name, sizeof(l->name) - 1);
    l->npoints = npoints;
    l->values = (PetscInt *)malloc((size_t)(npoints > 0 ? npoints : 1) * sizeof(PetscInt));
    for (int i = 0; i < npoints; i++) l->values[i] = -1;
    l->defval = -1;
    if (dm && dm->nlabels < SHIM_MAXLABEL) dm->labels[dm->nlabels++] = l;
    return l;
}
PetscErrorCode DMCreateLabel(DM dm, const char *name)
{
    if (!find_label(dm, name)) shim_label_new(dm, name, dm->ncells + dm->nfaces + dm->nbfaces);
    return 0;
}
PetscErrorCode DMGetLabel(DM dm, const char *name, DMLabel *l) { *l = find_label(dm, name); return 0; }
PetscErrorCode DMLabelCreate(MPI_Comm c, const char *name, DMLabel *l) { (void)c; (void)name; *l = NULL; return shim_unsupported("DMLabelCreate"); }
PetscErrorCode DMLabelSetDefaultValue(DMLabel l, PetscInt v) { if (l) l->defval = v; return 0; }
PetscErrorCode DMLabelSetValue(DMLabel l, PetscInt p, PetscInt v)
{
    if (!l || p < 0 || p >= l->npoints) return 1;
    l->values[p] = v;
    return 0;
}
PetscErrorCode DMLabelGetValue(DMLabel l, PetscInt p, PetscInt *v)
{
    if (!l || p < 0 || p >= l->npoints) { *v = -1; return 0; }
    *v = l->values[p] < 0 ? l->defval : l->values[p];
    return 0;
}
PetscErrorCode DMSetLabelValue(DM dm, const char *name, PetscInt p, PetscInt v) { return DMLabelSetValue(find_label(dm, name), p, v); }
PetscErrorCode DMGetLabelValue(DM dm, const char *name, PetscInt p, PetscInt *v) { return DMLabelGetValue(find_label(dm, name), p, v); }
PetscErrorCode DMLabelGetStratumIS(DMLabel l, PetscInt v, IS *is)
{
    *is = NULL;
    if (!l) return 0;
    int n = 0;
    for (int i = 0; i < l->npoints; i++) if (l->values[i] == v) n++;
    if (!n) return 0;
    IS s = (IS)calloc(1, sizeof(struct _p_IS));
    s->n = n;
    s->idx = (PetscInt *)malloc((size_t)n * sizeof(PetscInt));
    n = 0;
    for (int i = 0; i < l->npoints; i++) if (l->values[i] == v) s->idx[n++] = i;
    *is = s;
    return 0;
}
PetscErrorCode ISGetLocalSize(IS is, PetscInt *n) { *n = is ? is->n : 0; return 0; }
PetscErrorCode ISGetIndices(IS is, const PetscInt **i) { *i = is ? is->idx : NULL; return 0; }
PetscErrorCode ISRestoreIndices(IS is, const PetscInt **i) { (void)is; *i = NULL; return 0; }
PetscErrorCode ISGetMinMax(IS is, PetscInt *mn, PetscInt *mx)
{
    *mn = 0x7fffffff; *mx = -1;
    for (int i = 0; is && i < is->n; i++) {
        if (is->idx[i] < *mn) *mn = is->idx[i];
        if (is->idx[i] > *mx) *mx = is->idx[i];
    }
    return 0;
}
PetscErrorCode ISDestroy(IS *is) { if (*is) { free((*is)->idx); free(*is); } *is = NULL; return 0; }

/* ---------------- TS ---------------- */
PetscErrorCode TSGetSolution(TS ts, Vec *v) { *v = ts->sol; return 0; }
PetscErrorCode TSSetSolution(TS ts, Vec v) { ts->sol = v; return 0; }
PetscErrorCode TSGetApplicationContext(TS ts, void *ctx) { *(void **)ctx = ts->ctx; return 0; }
PetscErrorCode TSSetApplicationContext(TS ts, void *ctx) { ts->ctx = ctx; return 0; }
PetscErrorCode TSGetTime(TS ts, PetscReal *t) { *t = ts->t; return 0; }
PetscErrorCode TSSetTime(TS ts, PetscReal t) { ts->t = t; return 0; }
PetscErrorCode TSGetTimeStep(TS ts, PetscReal *dt) { *dt = ts->dt; return 0; }
PetscErrorCode TSSetTimeStep(TS ts, PetscReal dt) { ts->dt = dt; return 0; }
PetscErrorCode TSGetStepNumber(TS ts, PetscInt *s) { *s = ts->step; return 0; }
PetscErrorCode TSSetStepNumber(TS ts, PetscInt s) { ts->step = s; return 0; }
PetscErrorCode TSGetSolveTime(TS ts, PetscReal *t) { *t = ts->t; return 0; }

/* ---------------- everything the oracle never calls ---------------- */
#define SHIM_STUB(decl, name) PetscErrorCode decl { return shim_unsupported(name); }
SHIM_STUB(DMCreate(MPI_Comm c, DM *d), "DMCreate")
SHIM_STUB(DMSetType(DM d, DMType t), "DMSetType")
SHIM_STUB(DMSetFromOptions(DM d), "DMSetFromOptions")
SHIM_STUB(DMSetUp(DM d), "DMSetUp")
SHIM_STUB(DMConvert(DM d, DMType t, DM *o), "DMConvert")
SHIM_STUB(DMLocalizeCoordinates(DM d), "DMLocalizeCoordinates")
SHIM_STUB(DMDestroy(DM *d), "DMDestroy")
SHIM_STUB(DMClone(DM d, DM *o), "DMClone")
SHIM_STUB(DMSetField(DM d, PetscInt f, DMLabel l, PetscObject o), "DMSetField")
SHIM_STUB(DMCreateDS(DM d), "DMCreateDS")
SHIM_STUB(DMCopyDisc(DM a, DM b), "DMCopyDisc")
SHIM_STUB(DMCopyLabels(DM a, DM b, PetscCopyMode m, PetscBool x, DMCopyLabelsMode y), "DMCopyLabels")
SHIM_STUB(DMAdaptLabel(DM d, DMLabel l, DM *o), "DMAdaptLabel")
SHIM_STUB(DMForestSetTopology(DM d, const char *t), "DMForestSetTopology")
SHIM_STUB(DMForestSetInitialRefinement(DM d, PetscInt n), "DMForestSetInitialRefinement")
SHIM_STUB(DMForestSetMaximumRefinement(DM d, PetscInt n), "DMForestSetMaximumRefinement")
SHIM_STUB(DMForestSetMinimumRefinement(DM d, PetscInt n), "DMForestSetMinimumRefinement")
SHIM_STUB(DMForestSetPartitionOverlap(DM d, PetscInt n), "DMForestSetPartitionOverlap")
SHIM_STUB(DMForestSetAdaptivityForest(DM d, DM e), "DMForestSetAdaptivityForest")
SHIM_STUB(DMForestTransferVec(DM a, Vec b, DM c, Vec d, PetscBool e, PetscReal f), "DMForestTransferVec")
SHIM_STUB(PetscSFCreate(MPI_Comm c, PetscSF *s), "PetscSFCreate")
SHIM_STUB(PetscSFSetFromOptions(PetscSF s), "PetscSFSetFromOptions")
SHIM_STUB(PetscSFSetGraph(PetscSF s, PetscInt a, PetscInt b, PetscInt *c, PetscCopyMode d, PetscSFNode *e, PetscCopyMode f), "PetscSFSetGraph")
SHIM_STUB(PetscSFSetUp(PetscSF s), "PetscSFSetUp")
SHIM_STUB(PetscSFDestroy(PetscSF *s), "PetscSFDestroy")
SHIM_STUB(PetscSFReduceBegin(PetscSF s, MPI_Datatype t, const void *a, void *b, MPI_Op o), "PetscSFReduceBegin")
SHIM_STUB(PetscSFReduceEnd(PetscSF s, MPI_Datatype t, const void *a, void *b, MPI_Op o), "PetscSFReduceEnd")
SHIM_STUB(PetscSFBcastBegin(PetscSF s, MPI_Datatype t, const void *a, void *b, MPI_Op o), "PetscSFBcastBegin")
SHIM_STUB(PetscSFBcastEnd(PetscSF s, MPI_Datatype t, const void *a, void *b, MPI_Op o), "PetscSFBcastEnd")
SHIM_STUB(PetscFECreateDefault(MPI_Comm c, PetscInt a, PetscInt b, PetscBool x, const char *p, PetscInt q, PetscFE *f), "PetscFECreateDefault")
SHIM_STUB(PetscFEDestroy(PetscFE *f), "PetscFEDestroy")
PetscErrorCode PetscViewerVTKOpen(MPI_Comm c, const char *n, PetscFileMode m, PetscViewer *v)
{
    (void)c; (void)n; (void)m;
    *v = NULL;
    return shim_capture ? 0 : shim_unsupported("PetscViewerVTKOpen");
}
PetscErrorCode PetscViewerPushFormat(PetscViewer v, PetscViewerFormat f) { (void)v; (void)f; return 0; }
PetscErrorCode PetscViewerDestroy(PetscViewer *v) { *v = NULL; return 0; }
SHIM_STUB(TSCreate(MPI_Comm c, TS *t), "TSCreate")
SHIM_STUB(TSSetType(TS t, TSType y), "TSSetType")
SHIM_STUB(TSSetDM(TS t, DM d), "TSSetDM")
SHIM_STUB(TSSetRHSFunction(TS t, Vec v, PetscErrorCode (*f)(TS, PetscReal, Vec, Vec, void *), void *c), "TSSetRHSFunction")
SHIM_STUB(TSSetPostStep(TS t, PetscErrorCode (*f)(TS)), "TSSetPostStep")
SHIM_STUB(TSGetAdapt(TS t, TSAdapt *a), "TSGetAdapt")
SHIM_STUB(TSAdaptSetType(TSAdapt a, TSAdaptType t), "TSAdaptSetType")
SHIM_STUB(TSAdaptSetStepLimits(TSAdapt a, PetscReal x, PetscReal y), "TSAdaptSetStepLimits")
SHIM_STUB(TSSetTolerances(TS t, PetscReal a, Vec b, PetscReal c, Vec d), "TSSetTolerances")
SHIM_STUB(TSSetFromOptions(TS t), "TSSetFromOptions")
SHIM_STUB(TSSetMaxSteps(TS t, PetscInt n), "TSSetMaxSteps")
SHIM_STUB(TSSetMaxTime(TS t, PetscReal x), "TSSetMaxTime")
SHIM_STUB(TSSetExactFinalTime(TS t, TSExactFinalTimeOption o), "TSSetExactFinalTime")
SHIM_STUB(TSSolve(TS t, Vec v), "TSSolve")
SHIM_STUB(TSDestroy(TS *t), "TSDestroy")
