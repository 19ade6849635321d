/*
 * config.c - the reference's YAML configuration format read into a
 * cipher_problem and the rest of a run's settings (SetUpConfig,
 * src/init.c:104-1716).
 *
 * Every property is looked up the way the reference looks it up
 * (GetProperty on the file's event stream, yaml_lite.c), in the same order,
 * with the same defaults; numbers go through atof/atoi as there.  Where the
 * reference asserts, this loader returns CIPHER_E_ARG with the property
 * named.  Table orders are the reference parser's (binary pairs (ck<cj),
 * ternaries (ck<cj<ci), the calphad2sl (p:q) tables), which are also the
 * orders of cipher_problem.h.
 */
#define _POSIX_C_SOURCE 200809L
#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "cipher_b200.h"
#include "yaml_lite.h"

int cipher_host_set_error(int code, const char *msg);

#define CFG_MAXV 4096          /* values of one property (the reference keeps 100) */
#define CFG_PATH 1024

typedef struct {
    const yl_doc *d;
    const char *v[CFG_MAXV];
    int n;
    int rc;
    char msg[512];
    const char *basedir;
    int ncp, ndp, dim, npf;
    char comp[CIPHER_MAXCP][64];
} cfg_t;

static int cfg_fail(cfg_t *c, int code, const char *fmt, ...)
{
    if (c->rc) return c->rc;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(c->msg, sizeof(c->msg), fmt, ap);
    va_end(ap);
    c->rc = code;
    return code;
}

/* GetProperty: number of values of mapping/prop, values in c->v */
static int get(cfg_t *c, const char *mapping, const char *prop)
{
    c->n = yl_get(c->d, mapping, prop, c->v, CFG_MAXV);
    if (c->n > CFG_MAXV) {
        cfg_fail(c, CIPHER_E_ARG, "%s/%s: more than %d values", mapping, prop, CFG_MAXV);
        c->n = 0;
    }
    return c->n;
}

static const char *need_one(cfg_t *c, const char *mapping, const char *prop)
{
    if (get(c, mapping, prop) != 1) {
        cfg_fail(c, CIPHER_E_ARG, "%s/%s: expected one value, found %d", mapping, prop, c->n);
        return "0";
    }
    return c->v[0];
}

static double real_or(cfg_t *c, const char *mapping, const char *prop, double def)
{
    const int n = get(c, mapping, prop);
    if (!n) return def;
    if (n != 1) cfg_fail(c, CIPHER_E_ARG, "%s/%s: expected one value, found %d", mapping, prop, n);
    return atof(c->v[0]);
}

static int int_or(cfg_t *c, const char *mapping, const char *prop, int def)
{
    const int n = get(c, mapping, prop);
    if (!n) return def;
    if (n != 1) cfg_fail(c, CIPHER_E_ARG, "%s/%s: expected one value, found %d", mapping, prop, n);
    return atoi(c->v[0]);
}

/* n doubles of mapping/prop (exactly n, or absent when `optional`) */
static int reals(cfg_t *c, const char *mapping, const char *prop, int n, double *out, int optional)
{
    const int k = get(c, mapping, prop);
    if (!k && optional) return 0;
    if (k != n) return cfg_fail(c, CIPHER_E_ARG, "%s/%s: expected %d values, found %d", mapping, prop, n, k), 0;
    for (int i = 0; i < n; i++) out[i] = atof(c->v[i]);
    return n;
}

/* T-series at `mapping` (t_coefficient, t_exponent, tlnt_coefficient) */
static void tseries(cfg_t *c, const char *mapping, int with_log, cipher_tseries *t)
{
    memset(t, 0, sizeof(*t));
    const int n = get(c, mapping, "t_coefficient");
    if (n > CIPHER_MAXTSER) { cfg_fail(c, CIPHER_E_ARG, "%s: %d terms, at most %d", mapping, n, CIPHER_MAXTSER); return; }
    t->n = n;
    for (int i = 0; i < n; i++) t->coeff[i] = atof(c->v[i]);
    const int ne = get(c, mapping, "t_exponent");
    if (ne != n) { cfg_fail(c, CIPHER_E_ARG, "%s: %d exponents for %d coefficients", mapping, ne, n); return; }
    for (int i = 0; i < n; i++) t->exp[i] = atoi(c->v[i]);
    t->logcoeff = 0.0;
    if (with_log && get(c, mapping, "tlnt_coefficient")) t->logcoeff = atof(c->v[0]);
}

/* Redlich-Kister table at `mapping` (nrk, rk_<i>/..., index for ternaries) */
static void rk(cfg_t *c, const char *mapping, int with_index, cipher_rk *r)
{
    memset(r, 0, sizeof(*r));
    r->n = get(c, mapping, "nrk") ? atoi(c->v[0]) : 0;
    if (r->n < 0 || r->n > CIPHER_MAXRK) { cfg_fail(c, CIPHER_E_ARG, "%s/nrk: %d, at most %d", mapping, r->n, CIPHER_MAXRK); return; }
    char m[CFG_PATH];
    for (int k = 0; k < r->n; k++) {
        snprintf(m, sizeof(m), "%s/rk_%d", mapping, k);
        tseries(c, m, 0, &r->h[k]);
        if (with_index) r->i[k] = atoi(need_one(c, m, "index"));
    }
}

/* component mobilities of a material (src/init.c:371-413) */
static void mobilities(cfg_t *c, const char *mm, cipher_mobility *mob)
{
    char m[CFG_PATH];
    for (int a = 0; a < c->ncp; a++) {
        cipher_mobility *M = &mob[a];
        memset(M, 0, sizeof(*M));
        snprintf(m, sizeof(m), "%s/mobilityc/%s", mm, c->comp[a]);
        M->m0 = atof(need_one(c, m, "mobility0"));
        int b = 0;
        for (int j = 0; j < c->ncp; j++) {
            snprintf(m, sizeof(m), "%s/mobilityc/%s/unary_migration/%s", mm, c->comp[a], c->comp[j]);
            tseries(c, m, 0, &M->unary[j]);
            for (int i = j + 1; i < c->ncp; i++, b++) {
                snprintf(m, sizeof(m), "%s/mobilityc/%s/binary_migration/%s/%s", mm, c->comp[a], c->comp[j], c->comp[i]);
                rk(c, m, 0, &M->binary[b]);
            }
        }
    }
}

/* sources of a material or an interface (src/init.c:271-333) */
static void sources(cfg_t *c, const char *owner, int32_t *nsrc, cipher_source *src)
{
    char sm[CFG_PATH], am[CFG_PATH];
    snprintf(sm, sizeof(sm), "%s/sources", owner);
    const int n = get(c, sm, "activesources");
    if (n > CIPHER_MAXSRC) { cfg_fail(c, CIPHER_E_ARG, "%s/activesources: %d, at most %d", sm, n, CIPHER_MAXSRC); return; }
    char names[CIPHER_MAXSRC][256];
    for (int s = 0; s < n; s++) snprintf(names[s], sizeof(names[s]), "%s", c->v[s]);
    *nsrc = n;
    for (int s = 0; s < n; s++) {
        cipher_source *S = &src[s];
        memset(S, 0, sizeof(*S));
        snprintf(am, sizeof(am), "%s/%s", sm, names[s]);
        const char *model = need_one(c, am, "source");
        if (!strcmp(model, "sink")) {
            S->model = CIPHER_SOURCE_SINK;
            reals(c, am, "rate", c->ncp, S->rate, 1);
            reals(c, am, "ceq", c->ncp, S->ceq, 1);
        } else if (!strcmp(model, "random")) {
            S->model = CIPHER_SOURCE_RANDOM;
            /* the reference takes every value given here (src/init.c:1050-1056) */
            const int k = get(c, am, "fluctuation_amplitute");
            if (k > CIPHER_MAXCP) { cfg_fail(c, CIPHER_E_ARG, "%s/fluctuation_amplitute: %d values", am, k); return; }
            for (int i = 0; i < k; i++) S->amplitude[i] = atof(c->v[i]);
        } else {
            cfg_fail(c, CIPHER_E_ARG, "%s/source: unknown model '%s'", am, model);
            return;
        }
    }
}

static void material(cfg_t *c, const char *name, cipher_material *M)
{
    char mm[CFG_PATH], m[CFG_PATH];
    snprintf(mm, sizeof(mm), "material/%s", name);
    memset(M, 0, sizeof(*M));
    M->molarvolume = atof(need_one(c, mm, "molarvolume"));
    M->chempot_ex_kineticcoeff = real_or(c, mm, "chempot_ex_kineticcoeff", 0.0);
    sources(c, mm, &M->nsources, M->sources);
    const char *model = need_one(c, mm, "chemicalenergy");
    const int ncp = c->ncp;
    if (!strcmp(model, "none")) {
        M->model = CIPHER_CHEM_NONE;
        snprintf(m, sizeof(m), "%s/ref_enthalpy", mm);
        tseries(c, m, 0, &M->ref);
    } else if (!strcmp(model, "quadratic")) {
        M->model = CIPHER_CHEM_QUADRATIC;
        reals(c, mm, "c0", ncp, M->c0, 0);
        mobilities(c, mm, M->mobilityc);
        for (int a = 0; a < ncp; a++) {
            snprintf(m, sizeof(m), "%s/ceq/%s", mm, c->comp[a]);
            tseries(c, m, 0, &M->quad_ceq[a]);
        }
        snprintf(m, sizeof(m), "%s/ref_enthalpy", mm);
        tseries(c, m, 0, &M->ref);
        for (int a = 0; a < ncp; a++) {
            snprintf(m, sizeof(m), "%s/unary_enthalpy/%s", mm, c->comp[a]);
            tseries(c, m, 0, &M->unary[a]);
        }
        for (int a = 0; a < ncp; a++) {
            snprintf(m, sizeof(m), "%s/binary_enthalpy/%s", mm, c->comp[a]);
            tseries(c, m, 0, &M->quad_binary[a]);
        }
    } else if (!strcmp(model, "calphaddis")) {
        M->model = CIPHER_CHEM_CALPHADDIS;
        reals(c, mm, "c0", ncp, M->c0, 0);
        mobilities(c, mm, M->mobilityc);
        snprintf(m, sizeof(m), "%s/ref_enthalpy", mm);
        tseries(c, m, 0, &M->ref);
        for (int a = 0; a < ncp; a++) {
            snprintf(m, sizeof(m), "%s/unary_enthalpy/%s", mm, c->comp[a]);
            tseries(c, m, 1, &M->unary[a]);
        }
        int b = 0;
        for (int k = 0; k < ncp; k++)
            for (int j = k + 1; j < ncp; j++, b++) {
                snprintf(m, sizeof(m), "%s/binary_enthalpy/%s/%s", mm, c->comp[k], c->comp[j]);
                rk(c, m, 0, &M->binary[b]);
            }
        int t = 0;
        for (int k = 0; k < ncp; k++)
            for (int j = k + 1; j < ncp; j++)
                for (int i = j + 1; i < ncp; i++, t++) {
                    snprintf(m, sizeof(m), "%s/ternary_enthalpy/%s/%s/%s", mm, c->comp[k], c->comp[j], c->comp[i]);
                    rk(c, m, 1, &M->ternary[t]);
                }
    } else if (!strcmp(model, "calphad2sl")) {
        M->model = CIPHER_CHEM_CALPHAD2SL;
        reals(c, mm, "c0_p", ncp, M->c0, 0);
        reals(c, mm, "c0_q", ncp, M->c0 + ncp, 0);
        double pq[2] = {0.0, 0.0};
        reals(c, mm, "stochiometry", 2, pq, 0);
        M->p = pq[0];
        M->q = pq[1];
        if (!(fabs(M->p + M->q - 1.0) < CIPHER_TOL))
            cfg_fail(c, CIPHER_E_ARG, "%s/stochiometry: p + q = %g, not 1", mm, M->p + M->q);
        mobilities(c, mm, M->mobilityc);
        for (int p = 0; p < ncp; p++)
            for (int q = 0; q < ncp; q++) {
                snprintf(m, sizeof(m), "%s/unary_enthalpy/(%s:%s)", mm, c->comp[p], c->comp[q]);
                tseries(c, m, 1, &M->unary[p * ncp + q]);
            }
        int b = 0;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int q = 0; q < ncp; q++, b++) {
                    snprintf(m, sizeof(m), "%s/binary_enthalpy/(%s,%s:%s)", mm, c->comp[i], c->comp[j], c->comp[q]);
                    rk(c, m, 0, &M->binary[b]);
                }
        b = 0;
        for (int p = 0; p < ncp; p++)
            for (int i = 0; i < ncp; i++)
                for (int j = i + 1; j < ncp; j++, b++) {
                    snprintf(m, sizeof(m), "%s/binary_enthalpy/(%s:%s,%s)", mm, c->comp[p], c->comp[i], c->comp[j]);
                    rk(c, m, 0, &M->binaryq[b]);
                }
        int t = 0;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int k = j + 1; k < ncp; k++)
                    for (int q = 0; q < ncp; q++, t++) {
                        snprintf(m, sizeof(m), "%s/ternary_enthalpy/(%s,%s,%s:%s)", mm, c->comp[i], c->comp[j],
                                 c->comp[k], c->comp[q]);
                        rk(c, m, 0, &M->ternary[t]);
                    }
        t = 0;
        for (int p = 0; p < ncp; p++)
            for (int i = 0; i < ncp; i++)
                for (int j = i + 1; j < ncp; j++)
                    for (int k = j + 1; k < ncp; k++, t++) {
                        snprintf(m, sizeof(m), "%s/ternary_enthalpy/(%s:%s,%s,%s)", mm, c->comp[p], c->comp[i],
                                 c->comp[j], c->comp[k]);
                        rk(c, m, 0, &M->ternaryq[t]);
                    }
    } else {
        M->model = CIPHER_CHEM_NONE;   /* an unknown model is read as none (src/init.c:864-867) */
    }
    M->temperature0 = atof(need_one(c, mm, "temperature0"));
    snprintf(m, sizeof(m), "%s/specific_heat", mm);
    tseries(c, m, 0, &M->specific_heat);
    snprintf(m, sizeof(m), "%s/latent_heat", mm);
    tseries(c, m, 0, &M->latent_heat);
    snprintf(m, sizeof(m), "%s/tconductivity", mm);
    tseries(c, m, 0, &M->tconductivity);
}

/* anisotropy of an interface energy or mobility: values, and directions
 * normalised to unit length (src/init.c:1080-1102) */
static void anisotropy(cfg_t *c, const char *mapping, int32_t *n, double *dir, double *val)
{
    const int nv = get(c, mapping, "anisotropy_values");
    if (nv > CIPHER_MAXDIR) { cfg_fail(c, CIPHER_E_ARG, "%s/anisotropy_values: %d, at most %d", mapping, nv, CIPHER_MAXDIR); return; }
    *n = nv;
    for (int i = 0; i < nv; i++) val[i] = atof(c->v[i]);
    const int nd = get(c, mapping, "anisotropy_directions");
    if (!nd) return;
    if (nd != c->dim * nv) { cfg_fail(c, CIPHER_E_ARG, "%s/anisotropy_directions: %d values for %d directions", mapping, nd, nv); return; }
    for (int k = 0; k < nd; k += c->dim) {
        double norm = 0.0;
        for (int d = 0; d < c->dim; d++) {
            dir[k + d] = atof(c->v[k + d]);
            norm += dir[k + d] * dir[k + d];
        }
        norm = sqrt(norm);
        if (!(norm > 0.0)) { cfg_fail(c, CIPHER_E_ARG, "%s/anisotropy_directions: a zero direction", mapping); return; }
        for (int d = 0; d < c->dim; d++) dir[k + d] /= norm;
    }
}

static void interface(cfg_t *c, const char *name, cipher_interface *I)
{
    char im[CFG_PATH], m[CFG_PATH];
    snprintf(im, sizeof(im), "interface/%s", name);
    memset(I, 0, sizeof(*I));
    sources(c, im, &I->nsources, I->sources);
    snprintf(m, sizeof(m), "%s/mobility", im);
    I->mobility_m0 = atof(need_one(c, m, "m0"));
    snprintf(m, sizeof(m), "%s/mobility/activation_energy", im);
    tseries(c, m, 0, &I->mobility_activation);
    snprintf(m, sizeof(m), "%s/mobility", im);
    anisotropy(c, m, &I->mobility_naniso, I->mobility_aniso_dir, I->mobility_aniso_val);
    snprintf(m, sizeof(m), "%s/energy", im);
    I->energy_m0 = atof(need_one(c, m, "e0"));
    snprintf(m, sizeof(m), "%s/energy/activation_energy", im);
    tseries(c, m, 0, &I->energy_activation);
    snprintf(m, sizeof(m), "%s/energy", im);
    anisotropy(c, m, &I->energy_naniso, I->energy_aniso_dir, I->energy_aniso_val);
    if (get(c, im, "potential")) {
        I->has_potential = 1;
        reals(c, im, "potential", c->ndp, I->potential, 0);
    }
    if (get(c, im, "mobilityc")) {
        I->has_mobilityc = 1;
        reals(c, im, "mobilityc", c->ncp, I->mobilityc, 0);
    }
    I->width = atof(need_one(c, im, "width"));
}

static int bc_type(const char *s)
{
    if (!strcmp(s, "neumann")) return CIPHER_BC_NEUMANN;
    if (!strcmp(s, "dirichlet")) return CIPHER_BC_DIRICHLET;
    return CIPHER_BC_NONE;
}

static void boundary(cfg_t *c, const char *name, cipher_bc *B)
{
    char bm[CFG_PATH], m[CFG_PATH];
    snprintf(bm, sizeof(bm), "boundary/%s", name);
    memset(B, 0, sizeof(*B));
    B->boundaryid = atoi(need_one(c, bm, "boundary_id"));
    snprintf(m, sizeof(m), "%s/chem", bm);
    B->chem_bctype = CIPHER_BC_NONE;
    if (get(c, m, "type")) B->chem_bctype = bc_type(c->v[0]);
    const int nv = get(c, m, "value");
    if (B->chem_bctype != CIPHER_BC_NONE) {
        if (nv != c->ncp) { cfg_fail(c, CIPHER_E_ARG, "%s/value: expected %d values, found %d", m, c->ncp, nv); return; }
        for (int i = 0; i < nv; i++) {
            if (!strcmp(c->v[i], "*")) { B->chem_bcbool[i] = 0; B->chem_bcval[i] = 0.0; }
            else { B->chem_bcbool[i] = 1; B->chem_bcval[i] = atof(c->v[i]); }
        }
    }
    snprintf(m, sizeof(m), "%s/thermal", bm);
    B->thermal_bctype = CIPHER_BC_NONE;
    if (get(c, m, "type")) B->thermal_bctype = bc_type(c->v[0]);
    if (B->thermal_bctype != CIPHER_BC_NONE) B->thermal_bcval = atof(need_one(c, m, "value"));
}

static void nucleus(cfg_t *c, const char *name, cipher_nucleus *N)
{
    char nm[CFG_PATH];
    snprintf(nm, sizeof(nm), "nucleus/%s", name);
    memset(N, 0, sizeof(*N));
    const int nmat = get(c, nm, "matrix");
    if (nmat < 1 || nmat > 16) { cfg_fail(c, CIPHER_E_ARG, "%s/matrix: %d phases (1 to 16)", nm, nmat); return; }
    N->nmatrix = nmat;
    for (int i = 0; i < nmat; i++) N->matrix[i] = atoi(c->v[i]);
    /* the site check intersects sorted lists: keep the matrix sorted */
    for (int i = 1; i < nmat; i++)
        for (int j = i; j > 0 && N->matrix[j - 1] > N->matrix[j]; j--) {
            const int32_t t = N->matrix[j];
            N->matrix[j] = N->matrix[j - 1];
            N->matrix[j - 1] = t;
        }
    const int na = get(c, nm, "active_solutes");
    for (int a = 0; a < c->ncp; a++) N->active_solutes[a] = na ? 0 : 1;
    for (int i = 0; i < na; i++)
        for (int a = 0; a < c->ncp; a++)
            if (!strcmp(c->v[i], c->comp[a])) N->active_solutes[a] = 1;
    const char *model = need_one(c, nm, "nucleation_model");
    if (!strcmp(model, "cnt") || !strcmp(model, "thermal")) {
        const int thermal = !strcmp(model, "thermal");
        N->model = thermal ? CIPHER_NUC_THERMAL : CIPHER_NUC_CNT;
        if (thermal) {
            N->solvus_temperature_0 = atof(need_one(c, nm, "solvus_temperature_0"));
            if (get(c, nm, "solvus_temperature_c")) {
                N->has_solvus_c = 1;
                reals(c, nm, "solvus_temperature_c", c->ncp, N->solvus_temperature_c, 0);
            }
            N->enthalpy_fusion_0 = atof(need_one(c, nm, "enthalpy_fusion_0"));
            if (get(c, nm, "enthalpy_fusion_c")) {
                N->has_enthalpy_c = 1;
                reals(c, nm, "enthalpy_fusion_c", c->ncp, N->enthalpy_fusion_c, 0);
            }
        }
        N->gamma = atof(need_one(c, nm, "gamma"));
        N->shapefactor = real_or(c, nm, "shape_factor", 1.0);
        N->minsize = real_or(c, nm, "minsize", 0.0);
        N->atomicvolume = atof(need_one(c, nm, "atomic_volume"));
        N->lengthscale = atof(need_one(c, nm, "length_scale"));
        N->incubationtimemin = real_or(c, nm, "incubation_time", 0.0);
        N->liquidus = real_or(c, nm, "liquidus_temperature", CIPHER_LARGE);
    } else if (!strcmp(model, "constant")) {
        N->model = CIPHER_NUC_CONSTANT;
        N->nucleation_rate = atof(need_one(c, nm, "nucleation_rate"));
        N->incubationtimemin = real_or(c, nm, "incubation_time", 0.0);
    } else {
        N->model = CIPHER_NUC_NONE;
    }
}

/* ---------------- run-length mappings (src/init.c:1345-1712) ---------------- */

static char *read_file(const char *path, size_t *len)
{
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *b = n >= 0 ? (char *)malloc((size_t)n + 1) : NULL;
    if (b && fread(b, 1, (size_t)n, f) != (size_t)n) { free(b); b = NULL; }
    fclose(f);
    if (!b) return NULL;
    b[n] = 0;
    if (len) *len = (size_t)n;
    return b;
}

enum { RLE_PLAIN = 0, RLE_UPPER = 1 };

/* decode mappings/<prop> into out[total]: lines "N of V" (N copies of V-1),
 * "A to B" (A-1 .. B-1, either direction) and "V" (V-1; a line whose value
 * reads as 0 is skipped, as atoi() makes the reference skip it).  `maxv`
 * bounds V (0: no bound).  RLE_UPPER keeps only entries above the diagonal
 * of an n x n table (the interface mapping) and mirrors them below. */
static void rle(cfg_t *c, const char *prop, int32_t *out, int64_t total, int64_t maxv, int mode, int64_t ncol)
{
    if (!get(c, "mappings", prop)) { cfg_fail(c, CIPHER_E_ARG, "mappings/%s: missing", prop); return; }
    char *own = NULL;
    const char *text = c->v[0];
    /* a first line naming a .txt file holds the mapping */
    const char *nl = strchr(text, '\n');
    size_t l0 = nl ? (size_t)(nl - text) : strlen(text);
    char first[1024];
    snprintf(first, sizeof(first), "%.*s", (int)(l0 < sizeof(first) - 1 ? l0 : sizeof(first) - 1), text);
    if (strstr(first, ".txt")) {
        char path[2048];
        if (c->basedir && first[0] != '/') {
            snprintf(path, sizeof(path), "%s/%s", c->basedir, first);
            own = read_file(path, NULL);
        }
        if (!own) own = read_file(first, NULL);
        if (!own) { cfg_fail(c, CIPHER_E_ARG, "mappings/%s: cannot read %s", prop, first); return; }
        text = own;
    }
    int64_t k = 0;
    const char *s = text;
    int more = 0;
    while (*s) {
        const char *e = strchr(s, '\n');
        const size_t ll = e ? (size_t)(e - s) : strlen(s);
        if (ll == 0) { s = e ? e + 1 : s + ll; continue; }        /* strtok skips empty lines */
        if (k >= total) { more = 1; break; }
        char line[256];
        snprintf(line, sizeof(line), "%.*s", (int)(ll < sizeof(line) - 1 ? ll : sizeof(line) - 1), s);
        s = e ? e + 1 : s + ll;
        int64_t a = 0, b = 0, count = 0, step = 0;
        char sa[128], sb[128];
        if (strstr(line, "of")) {
            if (sscanf(line, "%127s of %127s", sa, sb) != 2) { cfg_fail(c, CIPHER_E_ARG, "mappings/%s: bad line '%s'", prop, line); break; }
            count = atoi(sa);
            a = b = atoi(sb);
            step = 0;
        } else if (strstr(line, "to")) {
            if (sscanf(line, "%127s to %127s", sa, sb) != 2) { cfg_fail(c, CIPHER_E_ARG, "mappings/%s: bad line '%s'", prop, line); break; }
            a = atoi(sa);
            b = atoi(sb);
            step = a < b ? 1 : -1;
            count = (a < b ? b - a : a - b) + 1;
        } else if (atoi(line)) {
            a = b = atoi(line);
            count = 1;
        } else {
            continue;
        }
        if (count < 0 || k + count > total) {
            cfg_fail(c, CIPHER_E_ARG, "mappings/%s: more than %lld entries", prop, (long long)total);
            break;
        }
        if (maxv > 0 && (a > maxv || b > maxv)) {
            cfg_fail(c, CIPHER_E_ARG, "mappings/%s: value %lld above %lld", prop, (long long)(a > b ? a : b), (long long)maxv);
            break;
        }
        for (int64_t j = 0; j < count; j++, k++) {
            const int32_t v = (int32_t)(a + step * j - 1);
            if (mode == RLE_UPPER) {
                const int64_t row = k / ncol, col = k % ncol;
                if (col > row) { out[k] = v; out[col * ncol + row] = v; }
            } else {
                out[k] = v;
            }
        }
    }
    free(own);
    if (c->rc) return;
    /* the reference asserts the count, and for all but the interface
     * mapping that no lines are left over */
    if (k != total) cfg_fail(c, CIPHER_E_ARG, "mappings/%s: %lld entries, expected %lld", prop, (long long)k, (long long)total);
    else if (more && mode != RLE_UPPER) cfg_fail(c, CIPHER_E_ARG, "mappings/%s: lines after %lld entries", prop, (long long)total);
}

/* ---------------- petscoptions ---------------- */

/* the value after `opt` among the options, or NULL */
static const char *option(const char *opts, const char *opt, char *val, size_t len)
{
    const size_t ol = strlen(opt);
    for (const char *s = opts; (s = strstr(s, opt)) != NULL; s += ol) {
        if ((s != opts && s[-1] != ' ') || (s[ol] != ' ' && s[ol] != 0)) continue;
        const char *v = s + ol;
        while (*v == ' ') v++;
        size_t n = 0;
        while (v[n] && v[n] != ' ' && n + 1 < len) { val[n] = v[n]; n++; }
        val[n] = 0;
        return val;
    }
    return NULL;
}

/* ---------------- the whole file ---------------- */

int cipher_output_field_parse(const char *name, int ncomponents, const char *const *components,
                              cipher_output_field *out)
{
    if (!name || !out) return CIPHER_E_ARG;
    memset(out, 0, sizeof(*out));
    snprintf(out->name, sizeof(out->name), "%s", name);
    /* the token before the first '_' (strtok_r(name, "_")) */
    char tok[256];
    const char *s = name;
    while (*s == '_') s++;
    size_t n = 0;
    while (s[n] && s[n] != '_' && n + 1 < sizeof(tok)) { tok[n] = s[n]; n++; }
    tok[n] = 0;
    int comp = 1 << 20;                 /* past every component: a zero field */
    for (int c = 0; c < ncomponents; c++)
        if (components && components[c] && !strcmp(components[c], tok)) { comp = c; break; }
    if (!strcmp(name, "phaseid")) out->kind = CIPHER_OUT_PHASEID;
    else if (!strcmp(name, "matid")) out->kind = CIPHER_OUT_MATID;
    else if (!strcmp(name, "interfaceid")) out->kind = CIPHER_OUT_INTERFACEID;
    else if (strstr(name, "_chempot")) { out->kind = CIPHER_OUT_CHEMPOT; out->index = comp; }
    else if (strstr(name, "_c")) { out->kind = CIPHER_OUT_COMP; out->index = comp; }
    else if (strstr(name, "_phi")) { out->kind = CIPHER_OUT_PHI; out->index = atoi(tok); }
    else if (!strcmp(name, "temperature")) out->kind = CIPHER_OUT_TEMPERATURE;
    else return cipher_host_set_error(CIPHER_E_ARG, "unknown output field");
    return CIPHER_OK;
}

void cipher_config_free(cipher_config *k)
{
    if (!k) return;
    cipher_problem_free(k->problem);
    free(k->voxelsite);
    free(k->sitephase);
    free(k->sitenucleus);
    free(k->nuclei);
    free(k->outputs);
    free(k);
}

static int names(cfg_t *c, const char *prop, int required, int maxn, char (*out)[64])
{
    const int n = get(c, "header", prop);
    if (required && n < 1) return cfg_fail(c, CIPHER_E_ARG, "header/%s: missing", prop), 0;
    if (n > maxn) return cfg_fail(c, CIPHER_E_ARG, "header/%s: %d names, at most %d", prop, n, maxn), 0;
    for (int i = 0; i < n; i++) {
        if (strlen(c->v[i]) >= 64) return cfg_fail(c, CIPHER_E_ARG, "header/%s: name too long", prop), 0;
        strcpy(out[i], c->v[i]);
    }
    return n;
}

int cipher_config_parse(const char *text, size_t len, const char *basedir, cipher_config **out)
{
    if (!text || !out) return cipher_host_set_error(CIPHER_E_ARG, "NULL argument");
    *out = NULL;
    char perr[256];
    yl_doc *d = yl_parse(text, len, perr, sizeof(perr));
    if (!d) {
        char m[320];
        snprintf(m, sizeof(m), "configuration: %s", perr[0] ? perr : "out of memory");
        return cipher_host_set_error(perr[0] ? CIPHER_E_ARG : CIPHER_E_NOMEM, m);
    }
    cfg_t *c = (cfg_t *)calloc(1, sizeof(cfg_t));
    cipher_config *k = (cipher_config *)calloc(1, sizeof(cipher_config));
    char (*matname)[64] = NULL, (*itfname)[64] = NULL, (*nucname)[64] = NULL, (*bcname)[64] = NULL;
    char (*outname)[64] = NULL;
    if (!c || !k) { free(c); free(k); yl_free(d); return cipher_host_set_error(CIPHER_E_NOMEM, "configuration"); }
    c->d = d;
    c->basedir = basedir;

    /* header (src/init.c:140-261) */
    const int dim = get(c, "header", "grid");
    if (dim < 1 || dim > 3) cfg_fail(c, CIPHER_E_ARG, "header/grid: %d values (1 to 3)", dim);
    int32_t res[3] = {1, 1, 1};
    double size[3] = {1.0, 1.0, 1.0};
    for (int i = 0; i < dim && !c->rc; i++) res[i] = atoi(c->v[i]);
    if (!c->rc) reals(c, "header", "size", dim, size, 0);
    const int npf = atoi(need_one(c, "header", "n_phases"));
    if (!c->rc && npf < 1) cfg_fail(c, CIPHER_E_ARG, "header/n_phases: %d", npf);
    int nsites = 0;
    if (get(c, "header", "n_sites")) {
        nsites = atoi(c->v[0]);
        if (c->n != 1 || nsites < 1) cfg_fail(c, CIPHER_E_ARG, "header/n_sites: expected one positive value");
    }
    const int maxnames = 1024;
    matname = calloc((size_t)maxnames, 64);
    itfname = calloc((size_t)maxnames, 64);
    nucname = calloc((size_t)maxnames, 64);
    bcname = calloc(CIPHER_MAXBC, 64);
    outname = calloc((size_t)maxnames, 64);
    if (!matname || !itfname || !nucname || !bcname || !outname) cfg_fail(c, CIPHER_E_NOMEM, "configuration");
    const int nmat = c->rc ? 0 : names(c, "materials", 1, maxnames, matname);
    const int nnuc = c->rc ? 0 : names(c, "nuclei", 0, maxnames, nucname);
    const int nf = c->rc ? 0 : names(c, "interfaces", 1, maxnames, itfname);
    const int ncp = c->rc ? 0 : names(c, "components", 1, CIPHER_MAXCP, c->comp);
    const int nbc = c->rc ? 0 : names(c, "boundaries", 0, CIPHER_MAXBC, bcname);
    const int nout = c->rc ? 0 : names(c, "outputs", 0, maxnames, outname);
    cipher_problem *p = NULL;
    if (!c->rc) {
        p = cipher_problem_new(dim, npf, ncp, nmat, nf);
        if (!p) cfg_fail(c, CIPHER_E_NOMEM, "configuration: problem tables");
    }
    k->problem = p;
    if (!c->rc) {
        c->ncp = ncp;
        c->ndp = ncp - 1;
        c->dim = dim;
        c->npf = npf;
        k->ncomponents = ncp;
        for (int i = 0; i < ncp; i++) strcpy(k->componentname[i], c->comp[i]);
        for (int i = 0; i < 3; i++) { p->resolution[i] = res[i]; p->size[i] = size[i]; p->periodic[i] = 0; }
        p->nbcs = nbc;
    }
    /* materials, nuclei, interfaces, boundaries (src/init.c:263-1216) */
    for (int m = 0; !c->rc && m < nmat; m++) material(c, matname[m], &p->material[m]);
    if (!c->rc && nnuc) {
        k->nnuclei = nnuc;
        k->nuclei = (cipher_nucleus *)calloc((size_t)nnuc, sizeof(cipher_nucleus));
        if (!k->nuclei) cfg_fail(c, CIPHER_E_NOMEM, "configuration: nuclei");
    }
    for (int n = 0; !c->rc && n < nnuc; n++) nucleus(c, nucname[n], &k->nuclei[n]);
    for (int i = 0; !c->rc && i < nf; i++) interface(c, itfname[i], &p->interface[i]);
    for (int b = 0; !c->rc && b < nbc; b++) boundary(c, bcname[b], &p->bcs[b]);

    /* solution parameters (src/init.c:1218-1325) */
    const char *sp = "solution_parameters";
    if (!c->rc) {
        const char *interp = need_one(c, sp, "interpolation");
        if (!strcmp(interp, "linear")) p->interpolation = CIPHER_INTERP_LINEAR;
        else if (!strcmp(interp, "quadratic")) p->interpolation = CIPHER_INTERP_QUADRATIC;
        else if (!strcmp(interp, "cubic")) p->interpolation = CIPHER_INTERP_CUBIC;
        else cfg_fail(c, CIPHER_E_ARG, "%s/interpolation: '%s'", sp, interp);
    }
    if (!c->rc) {
        const int nlc = get(c, sp, "time");
        if (nlc < 1 || nlc > CIPHER_MAXLC) cfg_fail(c, CIPHER_E_ARG, "%s/time: %d load cases (1 to %d)", sp, nlc, CIPHER_MAXLC);
        else {
            p->nloadcases = nlc;
            p->currentloadcase = 0;
            for (int i = 0; i < nlc; i++) p->time[i] = atof(c->v[i]);
            if (get(c, sp, "temperature_rate")) {
                p->has_temperature_rate = 1;
                reals(c, sp, "temperature_rate", nlc, p->temperature_rate, 0);
            }
        }
    }
    if (!c->rc) {
        p->timestep0 = real_or(c, sp, "timestep0", 1.0e-18);
        p->mintimestep = real_or(c, sp, "timestepmin", 1.0e-18);
        p->maxtimestep = real_or(c, sp, "timestepmax", p->time[0]);
        p->junctionpenalty = real_or(c, sp, "junctionpenalty", 1.0);
        if (get(c, sp, "initblocksize") != dim) cfg_fail(c, CIPHER_E_ARG, "%s/initblocksize: expected %d values", sp, dim);
        else for (int i = 0; i < dim; i++) k->initblocksize[i] = atoi(c->v[i]);
        for (int i = dim; i < 3; i++) k->initblocksize[i] = 1;
        k->initrefine = atoi(need_one(c, sp, "initrefine"));
        k->initcoarsen = atoi(need_one(c, sp, "initcoarsen"));
        k->maxnrefine = atoi(need_one(c, sp, "maxnrefine"));
        k->minnrefine = atoi(need_one(c, sp, "minnrefine"));
        k->amrinterval = atoi(need_one(c, sp, "amrinterval"));
        p->reltol = real_or(c, sp, "reltol", 1.0e-6);
        p->abstol = real_or(c, sp, "abstol", 1.0e-6);
        if (get(c, sp, "random_seed")) { k->has_random_seed = 1; k->random_seed = atoi(c->v[0]); }
        k->outputfreq = int_or(c, sp, "outputfreq", 1);
        snprintf(k->outfile, sizeof(k->outfile), "%s", get(c, sp, "outfile") ? c->v[0] : "output");
        snprintf(k->petscoptions, sizeof(k->petscoptions), "%s", get(c, sp, "petscoptions") ? c->v[0] : "");
        for (int i = 0; i < dim && !c->rc; i++) {
            const long long cells = (long long)k->initblocksize[i] << (k->initrefine > 0 ? k->initrefine : 0);
            if (k->initrefine < 0 || k->initrefine > 24 || cells != res[i])
                cfg_fail(c, CIPHER_E_ARG, "%s: initblocksize[%d] * 2^initrefine = %lld, grid %d", sp, i, cells, res[i]);
        }
        p->gradient_calculation = int_or(c, sp, "gradient_calculation", 0);
        if (p->gradient_calculation < 0 || p->gradient_calculation > 1)
            cfg_fail(c, CIPHER_E_ARG, "%s/gradient_calculation: %d (0 or 1)", sp, p->gradient_calculation);
        k->max_phase_neighbours = int_or(c, sp, "max_phase_neighbours", CIPHER_MAXAP);
    }
    if (!c->rc) {
        char v[64];
        snprintf(k->rk_type, sizeof(k->rk_type), "%s", option(k->petscoptions, "-ts_rk_type", v, sizeof(v)) ? v : "3bs");
        if (option(k->petscoptions, "-dm_p4est_brick_periodicity", v, sizeof(v))) {
            char *save = NULL;
            int d = 0;
            for (char *t = strtok_r(v, ",", &save); t && d < 3; t = strtok_r(NULL, ",", &save), d++)
                p->periodic[d] = !strcmp(t, "1") || !strcmp(t, "true") || !strcmp(t, "yes");
        }
        if (k->max_phase_neighbours < 1 || k->max_phase_neighbours > CIPHER_MAXAP)
            cfg_fail(c, CIPHER_E_ARG, "%s/max_phase_neighbours: %d (1 to %d here)", sp, k->max_phase_neighbours, CIPHER_MAXAP);
        else cipher_problem_set_cap(p, k->max_phase_neighbours);
    }

    /* mappings (src/init.c:1345-1712) */
    const int64_t total = (int64_t)res[0] * res[1] * res[2];
    if (!c->rc) {
        rle(c, "phase_material_mapping", p->phasematerialmapping, npf, nmat, RLE_PLAIN, 0);
        p->voxelphase = (int32_t *)calloc((size_t)total, sizeof(int32_t));
        if (!p->voxelphase) cfg_fail(c, CIPHER_E_NOMEM, "configuration: voxel map");
    }
    if (!c->rc) rle(c, "voxel_phase_mapping", p->voxelphase, total, npf, RLE_PLAIN, 0);
    if (!c->rc) {
        for (int64_t i = 0; i < (int64_t)npf * npf; i++) p->interfacelist[i] = 0;
        rle(c, "interface_mapping", p->interfacelist, (int64_t)npf * npf, nf, RLE_UPPER, npf);
    }
    if (!c->rc && nsites) {
        k->nsites = nsites;
        k->sitenucleus = (int32_t *)calloc((size_t)nsites, sizeof(int32_t));
        k->sitephase = (int32_t *)calloc((size_t)nsites, sizeof(int32_t));
        k->voxelsite = (int32_t *)calloc((size_t)total, sizeof(int32_t));
        if (!k->sitenucleus || !k->sitephase || !k->voxelsite) cfg_fail(c, CIPHER_E_NOMEM, "configuration: sites");
        if (!c->rc) rle(c, "site_nucleus_mapping", k->sitenucleus, nsites, nnuc, RLE_PLAIN, 0);
        if (!c->rc) rle(c, "site_phase_mapping", k->sitephase, nsites, npf, RLE_PLAIN, 0);
        if (!c->rc) rle(c, "voxel_site_mapping", k->voxelsite, total, 0, RLE_PLAIN, 0);
        /* the site label is the mapped value minus one and site s is the
         * label s+1 (src/cipher.c:1308, 736): value 1 marks no site */
        for (int64_t i = 0; !c->rc && i < total; i++) {
            const int32_t s = k->voxelsite[i] - 1;
            k->voxelsite[i] = (s >= 0 && s < nsites) ? s : -1;
        }
    }
    if (!c->rc) {
        for (int64_t i = 0; i < total; i++)
            if (p->voxelphase[i] < 0) { cfg_fail(c, CIPHER_E_ARG, "mappings/voxel_phase_mapping: phase %d", p->voxelphase[i] + 1); break; }
    }
    /* outputs */
    if (!c->rc && nout) {
        k->noutputs = nout;
        k->outputs = (cipher_output_field *)calloc((size_t)nout, sizeof(cipher_output_field));
        if (!k->outputs) cfg_fail(c, CIPHER_E_NOMEM, "configuration: outputs");
        const char *cn[CIPHER_MAXCP];
        for (int i = 0; i < ncp; i++) cn[i] = c->comp[i];
        for (int o = 0; !c->rc && o < nout; o++)
            if (cipher_output_field_parse(outname[o], ncp, cn, &k->outputs[o]))
                cfg_fail(c, CIPHER_E_ARG, "header/outputs: unknown field '%s'", outname[o]);
    }
    if (!c->rc && cipher_problem_finalize(p)) cfg_fail(c, CIPHER_E_ARG, "configuration: problem tables");

    int rc = c->rc;
    if (rc) {
        cipher_host_set_error(rc, c->msg);
        cipher_config_free(k);
        k = NULL;
    }
    free(matname); free(itfname); free(nucname); free(bcname); free(outname);
    free(c);
    yl_free(d);
    *out = k;
    return rc;
}

int cipher_config_load(const char *path, cipher_config **out)
{
    if (!path || !out) return cipher_host_set_error(CIPHER_E_ARG, "NULL argument");
    *out = NULL;
    size_t len = 0;
    char *text = read_file(path, &len);
    if (!text) {
        char m[1100];
        snprintf(m, sizeof(m), "configuration file %s cannot be read", path);
        return cipher_host_set_error(CIPHER_E_ARG, m);
    }
    char dir[1024];
    snprintf(dir, sizeof(dir), "%s", path);
    char *slash = strrchr(dir, '/');
    if (slash) *slash = 0;
    else strcpy(dir, ".");
    const int rc = cipher_config_parse(text, len, dir, out);
    free(text);
    return rc;
}

/* ---------------- JSON view ---------------- */

typedef struct {
    char *out;
    size_t cap, n;
} jbuf;

static void jput(jbuf *b, const char *s, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        if (b->n + 1 < b->cap) b->out[b->n] = s[i];
        b->n++;
    }
}

static void jstr(jbuf *b, const char *s)
{
    jput(b, "\"", 1);
    for (; *s; s++) {
        const unsigned char ch = (unsigned char)*s;
        char esc[8];
        if (ch == '"' || ch == '\\') { esc[0] = '\\'; esc[1] = (char)ch; jput(b, esc, 2); }
        else if (ch == '\n') jput(b, "\\n", 2);
        else if (ch == '\t') jput(b, "\\t", 2);
        else if (ch == '\r') jput(b, "\\r", 2);
        else if (ch < 0x20) { snprintf(esc, sizeof(esc), "\\u%04x", ch); jput(b, esc, 6); }
        else jput(b, (const char *)&ch, 1);
    }
    jput(b, "\"", 1);
}

static void jnode(jbuf *b, const yl_node *n)
{
    if (n->kind == YL_SCALAR) { jstr(b, n->value); return; }
    const int map = n->kind == YL_MAPPING;
    jput(b, map ? "{" : "[", 1);
    for (int i = 0; i < n->n; i++) {
        if (i) jput(b, ",", 1);
        if (map) { jstr(b, n->keys[i]); jput(b, ":", 1); }
        jnode(b, n->kids[i]);
    }
    jput(b, map ? "}" : "]", 1);
}

int cipher_yaml_to_json(const char *text, size_t len, char *out, size_t outlen, size_t *needed)
{
    if (!text) return cipher_host_set_error(CIPHER_E_ARG, "NULL argument");
    char perr[256];
    yl_doc *d = yl_parse(text, len, perr, sizeof(perr));
    if (!d) return cipher_host_set_error(CIPHER_E_ARG, perr[0] ? perr : "out of memory");
    jbuf b = {out, out ? outlen : 0, 0};
    if (d->root) jnode(&b, d->root);
    else jput(&b, "null", 4);
    if (out && outlen) out[b.n < outlen ? b.n : outlen - 1] = 0;
    if (needed) *needed = b.n + 1;
    yl_free(d);
    return (out && b.n + 1 > outlen) ? cipher_host_set_error(CIPHER_E_ARG, "output buffer too small") : CIPHER_OK;
}
