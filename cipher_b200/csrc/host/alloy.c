/*
 * alloy.c - seeded synthetic alloy problems: two matrix grains with
 * spherical precipitates, CALPHAD (or quadratic) free energies with
 * random coefficients, and optional segregation, interface mobility factors,
 * T-dependent interface properties, heat, solute sinks, walls and a cooling
 * rate.  It fills the same tables the reference reads from its YAML input
 * (src/init.c:320-1260) so every model branch of the RHS can be exercised.
 *
 * Units: lengths in cells (cell size 1), energies in J/mol over a molar
 * volume of 1e-5, T = 700 K.  Coefficient ranges follow the magnitudes of
 * the reference's shipped alloy inputs: endmember energies a + b*T with
 * a ~ U[-5e4,-1e4], b ~ U[-20,20]; Redlich-Kister terms ~ U[-2e4,2e4];
 * solute fractions 0.02 / 0.01 with 1 % noise; diffusivities log-uniform
 * over two decades.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "cipher_problem.h"
#include "cipher_b200.h"

static double uni(uint64_t *s, double lo, double hi) { return lo + (hi - lo) * cipher_rand_uniform(s); }

static void tser_const(cipher_tseries *t, double v)
{
    memset(t, 0, sizeof(*t));
    t->n = 1;
    t->exp[0] = 0;
    t->coeff[0] = v;
}

/* a + b*T (+ c*T*ln T) */
static void tser_linear(cipher_tseries *t, uint64_t *s, int with_log)
{
    memset(t, 0, sizeof(*t));
    t->n = 2;
    t->exp[0] = 0;
    t->coeff[0] = uni(s, -5.0e4, -1.0e4);
    t->exp[1] = 1;
    t->coeff[1] = uni(s, -20.0, 20.0);
    if (with_log) t->logcoeff = uni(s, -1.0, 1.0);
}

static void rk_random(cipher_rk *rk, uint64_t *s, int n, double amp, int ncomp)
{
    memset(rk, 0, sizeof(*rk));
    rk->n = n;
    for (int r = 0; r < n; r++) {
        tser_const(&rk->h[r], uni(s, -amp, amp));
        rk->i[r] = (int32_t)(cipher_rand_uniform(s) * ncomp) % ncomp;
    }
}

/* fractions of ncp components: solutes 0.02, 0.01, 0.01, ... with 1 % noise,
 * the last component the balance; `shift` moves solute to the first one */
static void fractions(double *c, int ncp, uint64_t *s, double shift)
{
    double sum = 0.0;
    for (int k = 0; k < ncp - 1; k++) {
        double base = k == 0 ? 0.02 + shift : 0.01;
        c[k] = base * (1.0 + uni(s, -0.01, 0.01));
        sum += c[k];
    }
    c[ncp - 1] = 1.0 - sum;
}

static void mobilities(cipher_material *m, int ncp, uint64_t *s)
{
    for (int k = 0; k < ncp; k++) {
        cipher_mobility *mob = &m->mobilityc[k];
        memset(mob, 0, sizeof(*mob));
        mob->m0 = pow(10.0, uni(s, -1.0, 1.0));
        for (int j = 0; j < ncp; j++) tser_const(&mob->unary[j], uni(s, -1.0e3, 1.0e3));
        int b = 0;
        for (int j = 0; j < ncp; j++)
            for (int i = j + 1; i < ncp; i++, b++) rk_random(&mob->binary[b], s, 1, 1.0e3, ncp);
    }
}

static void material_model(cipher_material *m, int model, int ncp, uint64_t *s, double p, double shift)
{
    m->model = model;
    m->molarvolume = 1.0e-5;
    m->temperature0 = 700.0;
    tser_const(&m->ref, uni(s, -1.0e3, 1.0e3));
    if (model == CIPHER_CHEM_CALPHAD2SL) {
        m->p = p;
        m->q = 1.0 - p;
        for (int a = 0; a < ncp * ncp; a++) tser_linear(&m->unary[a], s, 1);
        int k = 0;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int q = 0; q < ncp; q++, k++) rk_random(&m->binary[k], s, 2, 2.0e4, ncp);
        k = 0;
        for (int pp = 0; pp < ncp; pp++)
            for (int i = 0; i < ncp; i++)
                for (int j = i + 1; j < ncp; j++, k++) rk_random(&m->binaryq[k], s, 1, 2.0e4, ncp);
        k = 0;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int l = j + 1; l < ncp; l++)
                    for (int q = 0; q < ncp; q++, k++) rk_random(&m->ternary[k], s, 1, 1.0e4, ncp);
        k = 0;
        for (int pp = 0; pp < ncp; pp++)
            for (int i = 0; i < ncp; i++)
                for (int j = i + 1; j < ncp; j++)
                    for (int l = j + 1; l < ncp; l++, k++) rk_random(&m->ternaryq[k], s, 1, 1.0e4, ncp);
        fractions(m->c0, ncp, s, shift);
        /* second sublattice: mostly the last component */
        double sum = 0.0;
        for (int c = 0; c < ncp - 1; c++) { m->c0[ncp + c] = 0.005 * (1.0 + uni(s, -0.01, 0.01)); sum += m->c0[ncp + c]; }
        m->c0[2 * ncp - 1] = 1.0 - sum;
    } else if (model == CIPHER_CHEM_CALPHADDIS) {
        for (int c = 0; c < ncp; c++) tser_linear(&m->unary[c], s, 1);
        int k = 0;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++, k++) rk_random(&m->binary[k], s, 3, 2.0e4, ncp);
        k = 0;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int l = j + 1; l < ncp; l++, k++) {
                    rk_random(&m->ternary[k], s, 1, 1.0e4, ncp);
                    /* the index picks one of the three components */
                    int pick = (int)(cipher_rand_uniform(s) * 3) % 3;
                    m->ternary[k].i[0] = pick == 0 ? i : (pick == 1 ? j : l);
                }
        fractions(m->c0, ncp, s, shift);
    } else {
        fractions(m->c0, ncp, s, shift);
        for (int c = 0; c < ncp; c++) {
            tser_const(&m->unary[c], uni(s, -1.0e3, 1.0e3));
            tser_const(&m->quad_ceq[c], m->c0[c]);
            tser_const(&m->quad_binary[c], uni(s, 1.0e5, 1.0e6));
        }
    }
    mobilities(m, ncp, s);
}

int cipher_problem_alloy(int dim, const int32_t *res, int model, int ncp, int nprecip, int cap, uint64_t seed,
                         unsigned features, cipher_problem **out)
{
    if (!out) return CIPHER_E_ARG;
    *out = NULL;
    if (dim < 1 || dim > 3 || ncp < 2 || ncp > CIPHER_MAXCP || nprecip < 0 || nprecip > 4000) return CIPHER_E_ARG;
    if (model != CIPHER_CHEM_QUADRATIC && model != CIPHER_CHEM_CALPHADDIS && model != CIPHER_CHEM_CALPHAD2SL)
        return CIPHER_E_ARG;
    for (int d = 0; d < dim; d++)
        if (res[d] < 1) return CIPHER_E_ARG;
    const int npf = 2 + nprecip;
    cipher_problem *p = cipher_problem_new(dim, npf, ncp, 2, 3);
    if (!p) return CIPHER_E_NOMEM;
    uint64_t s = seed ^ 0xA5A5A5A55A5A5A5AULL;
    for (int d = 0; d < dim; d++) {
        p->resolution[d] = res[d];
        p->size[d] = (double)res[d];
        p->periodic[d] = 1;
    }
    int rc = cipher_problem_set_cap(p, cap);
    if (rc) { cipher_problem_free(p); return rc; }

    /* materials: 0 = matrix, 1 = precipitate */
    int mmodel = (features & CIPHER_ALLOY_MIXED_MODELS) ? CIPHER_CHEM_CALPHADDIS : model;
    int pmodel = (features & CIPHER_ALLOY_MIXED_MODELS) ? CIPHER_CHEM_CALPHAD2SL : model;
    material_model(&p->material[0], mmodel, ncp, &s, 0.5, 0.0);
    material_model(&p->material[1], pmodel, ncp, &s, 2.0 / 3.0, 0.1);
    p->material[0].chempot_ex_kineticcoeff = 1.0;
    p->material[1].chempot_ex_kineticcoeff = 0.5;
    if (features & CIPHER_ALLOY_THERMAL) {
        for (int m = 0; m < 2; m++) {
            tser_const(&p->material[m].specific_heat, 2.3e6 * (1.0 + 0.1 * m));
            tser_const(&p->material[m].tconductivity, 6.7e6 * (1.0 - 0.2 * m));
            tser_const(&p->material[m].latent_heat, m == 1 ? 1.0e8 : 0.0);
        }
    }
    if (features & CIPHER_ALLOY_SOURCES) {
        cipher_material *m = &p->material[1];
        m->nsources = 1;
        m->sources[0].model = CIPHER_SOURCE_SINK;
        for (int c = 0; c < ncp; c++) {
            m->sources[0].rate[c] = uni(&s, 0.0, 1.0e-3);
            m->sources[0].ceq[c] = m->c0[c];
        }
    }

    /* interfaces: 0 = grain boundary, 1 = matrix/precipitate, 2 = precipitate/precipitate */
    const double e0[3] = {3.0e8, 5.0e8, 4.0e8}, m0[3] = {8.0e-11, 5.0e-11, 2.0e-11};
    for (int i = 0; i < 3; i++) {
        cipher_interface *itf = &p->interface[i];
        itf->width = 4.0;
        itf->energy_m0 = e0[i];
        itf->mobility_m0 = m0[i];
        if ((features & CIPHER_ALLOY_ACTIVATION) && i < 2) {
            tser_const(&itf->energy_activation, uni(&s, -2.0e3, 2.0e3));
            tser_const(&itf->mobility_activation, uni(&s, -2.0e4, -5.0e3));
        }
        if ((features & CIPHER_ALLOY_SEGREGATION) && i < 2) {
            itf->has_potential = 1;
            for (int c = 0; c < ncp - 1; c++) itf->potential[c] = uni(&s, -2.0e7, 2.0e7);
        }
        if ((features & CIPHER_ALLOY_ITF_MOBILITY) && i == 1) {
            itf->has_mobilityc = 1;
            for (int c = 0; c < ncp; c++) itf->mobilityc[c] = uni(&s, -5.0e3, 5.0e3);
        }
        if ((features & CIPHER_ALLOY_SOURCES) && i == 0) {
            itf->nsources = 1;
            itf->sources[0].model = CIPHER_SOURCE_SINK;
            for (int c = 0; c < ncp; c++) {
                itf->sources[0].rate[c] = uni(&s, 0.0, 1.0e-3);
                itf->sources[0].ceq[c] = p->material[0].c0[c];
            }
        }
    }
    for (int a = 0; a < npf; a++) {
        p->phasematerialmapping[a] = a < 2 ? 0 : 1;
        for (int b = 0; b < npf; b++) {
            int ka = a < 2, kb = b < 2;
            p->interfacelist[a * npf + b] = (ka && kb) ? 0 : ((ka || kb) ? 1 : 2);
        }
    }
    if (features & CIPHER_ALLOY_TEMP_RATE) {
        p->has_temperature_rate = 1;
        p->temperature_rate[0] = -1.0;
    }
    if (features & CIPHER_ALLOY_WALLS) {
        p->periodic[0] = 0;
        p->nbcs = 2;
        cipher_bc *lo = &p->bcs[0], *hi = &p->bcs[1];
        lo->boundaryid = 1;
        lo->chem_bctype = CIPHER_BC_NEUMANN;
        lo->thermal_bctype = CIPHER_BC_DIRICHLET;
        lo->thermal_bcval = 690.0;
        hi->boundaryid = 2;
        hi->chem_bctype = CIPHER_BC_DIRICHLET;
        hi->thermal_bctype = CIPHER_BC_NEUMANN;
        hi->thermal_bcval = 1.0e-3;
        for (int c = 0; c < ncp - 1; c++) {
            lo->chem_bcbool[c] = (int8_t)(c != 1);
            lo->chem_bcval[c] = uni(&s, -1.0e7, 1.0e7);
            hi->chem_bcbool[c] = 1;
            hi->chem_bcval[c] = uni(&s, -1.0e9, 1.0e9);
        }
    }
    p->reltol = p->abstol = 1.0e-4;
    p->time[0] = 1.0e3;
    p->maxtimestep = 1.0;

    /* voxel map: two matrix grains (Voronoi), then spherical precipitates */
    long total = 1;
    for (int d = 0; d < dim; d++) total *= res[d];
    p->voxelphase = (int32_t *)malloc((size_t)total * sizeof(int32_t));
    double *cen = (double *)malloc((size_t)(nprecip > 0 ? nprecip : 1) * 3 * sizeof(double));
    if (!p->voxelphase || !cen) { free(cen); cipher_problem_free(p); return CIPHER_E_NOMEM; }
    rc = cipher_voronoi(dim, res, 2, seed, p->voxelphase, NULL);
    if (rc) { free(cen); cipher_problem_free(p); return rc; }
    int rmin = res[0];
    for (int d = 1; d < dim; d++) rmin = res[d] < rmin ? res[d] : rmin;
    double rad = rmin / 8.0 < 2.0 ? 2.0 : rmin / 8.0;
    for (int k = 0; k < nprecip; k++)
        for (int d = 0; d < 3; d++) cen[3 * k + d] = d < dim ? uni(&s, 0.0, (double)res[d]) : 0.5;
    int r3[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) r3[d] = res[d];
    for (long g = 0; g < total; g++) {
        int x[3] = {(int)(g % r3[0]), (int)((g / r3[0]) % r3[1]), (int)(g / ((long)r3[0] * r3[1]))};
        for (int k = 0; k < nprecip; k++) {
            double d2 = 0.0;
            for (int d = 0; d < dim; d++) {
                double v = x[d] + 0.5 - cen[3 * k + d];
                if (v > 0.5 * r3[d]) v -= r3[d];
                if (v < -0.5 * r3[d]) v += r3[d];
                d2 += v * v;
            }
            if (d2 <= rad * rad) { p->voxelphase[g] = 2 + k; break; }
        }
    }
    free(cen);
    rc = cipher_problem_finalize(p);
    if (rc) { cipher_problem_free(p); return rc; }
    *out = p;
    return 0;
}
