/*
 * oracle_ts.c - CPU restatement of the library's explicit RK time stepper
 * (cipher_b200/csrc/cuda/ts.cu) over the oracle RHS and PostStep.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference steps with PETSc's TSRK and TSADAPTDSP (src/cipher.c:
 * 1097-1115), which are not vendored: the stepper is a project-written
 * restatement from the published methods, and this file restates it once
 * more on the CPU so that device trajectories can be checked.  Everything
 * is done in the same operation order as the device, including the error
 * norm's reduction tree (blocks of 2048 cells x 256 threads, a shuffle-down
 * tree per warp, warps in order, then 1024 threads over the partials), so
 * an FP64 trajectory is expected to match the device's bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "cipher_b200.h"

#define TS_THREADS 256
#define TS_CELLS_PER_BLOCK 2048
#define TS_MAXSTAGES 4

typedef struct oracle_ts {
    const cipher_problem *p;
    const cipher_mesh *m;
    cipher_ts_opts o;
    int ns, eorder;
    double A[TS_MAXSTAGES][TS_MAXSTAGES], b[TS_MAXSTAGES], bh[TS_MAXSTAGES], c[TS_MAXSTAGES];
    cipher_aos_layout L;
    int ncells, ndof, nplanes;
    int *plane_col;                 /* AoS column of each state plane, device plane order */
    double *K[TS_MAXSTAGES], *Y, *E;
    double dt, e_prev;
    int have_prev;
    cipher_ts_stats st;
} oracle_ts;

static int ts_tableau(oracle_ts *t, int scheme)
{
    memset(t->A, 0, sizeof(t->A));
    memset(t->b, 0, sizeof(t->b));
    memset(t->bh, 0, sizeof(t->bh));
    memset(t->c, 0, sizeof(t->c));
    if (scheme == CIPHER_TS_RK1FE) {
        t->ns = 1; t->eorder = 0;
        t->b[0] = 1.0;
    } else if (scheme == CIPHER_TS_RK2A) {
        t->ns = 2; t->eorder = 1;
        t->A[1][0] = 1.0;
        t->b[0] = 0.5; t->b[1] = 0.5;
        t->bh[0] = 1.0; t->bh[1] = 0.0;
        t->c[1] = 1.0;
    } else if (scheme == CIPHER_TS_RK3BS) {
        t->ns = 4; t->eorder = 2;
        t->A[1][0] = 1.0 / 2.0;
        t->A[2][1] = 3.0 / 4.0;
        t->A[3][0] = 2.0 / 9.0; t->A[3][1] = 1.0 / 3.0; t->A[3][2] = 4.0 / 9.0;
        t->b[0] = 2.0 / 9.0; t->b[1] = 1.0 / 3.0; t->b[2] = 4.0 / 9.0; t->b[3] = 0.0;
        t->bh[0] = 7.0 / 24.0; t->bh[1] = 1.0 / 4.0; t->bh[2] = 1.0 / 3.0; t->bh[3] = 1.0 / 8.0;
        t->c[1] = 1.0 / 2.0; t->c[2] = 3.0 / 4.0; t->c[3] = 1.0;
    } else {
        return 0;
    }
    return 1;
}

void oracle_ts_destroy(oracle_ts *t)
{
    if (!t) return;
    for (int j = 0; j < TS_MAXSTAGES; j++) free(t->K[j]);
    free(t->Y);
    free(t->E);
    free(t->plane_col);
    free(t);
}

oracle_ts *oracle_ts_create(const cipher_problem *p, const cipher_mesh *m, const cipher_ts_opts *o)
{
    if (m->ncells != m->nowned) return NULL;
    oracle_ts *t = (oracle_ts *)calloc(1, sizeof(oracle_ts));
    if (!t) return NULL;
    t->p = p;
    t->m = m;
    t->o = *o;
    if (!ts_tableau(t, o->scheme)) { free(t); return NULL; }
    t->L = or_aos_layout(p);
    t->ncells = m->ncells;
    t->ndof = t->L.ndof;
    t->nplanes = t->L.pf_size + t->L.dp_size + t->L.ex_size + 1;
    t->plane_col = (int *)malloc((size_t)t->nplanes * sizeof(int));
    size_t nb = (size_t)t->ncells * t->ndof * sizeof(double);
    for (int j = 0; j < t->ns; j++) t->K[j] = (double *)calloc(1, nb);
    t->Y = (double *)calloc(1, nb);
    t->E = (double *)calloc(1, nb);
    if (!t->plane_col || !t->Y || !t->E) { oracle_ts_destroy(t); return NULL; }
    for (int j = 0; j < t->ns; j++)
        if (!t->K[j]) { oracle_ts_destroy(t); return NULL; }
    int k = 0;
    for (int g = 0; g < t->L.pf_size; g++) t->plane_col[k++] = t->L.pf_offset + g;
    for (int d = 0; d < t->L.dp_size; d++) t->plane_col[k++] = t->L.dp_offset + d;
    for (int q = 0; q < t->L.ex_size; q++) t->plane_col[k++] = t->L.ex_offset + q;
    t->plane_col[k++] = t->L.tm_offset;
    double dt = o->dt0 < o->dtmin ? o->dtmin : (o->dt0 > o->dtmax ? o->dtmax : o->dt0);
    t->dt = dt;
    t->st.dt = dt;
    return t;
}

/* the device's __shfl_down_sync tree over one warp; returns lane 0 */
static double warp_tree(double *v)
{
    double w[32];
    for (int o = 16; o > 0; o >>= 1) {
        for (int i = 0; i < 32; i++) w[i] = v[i] + (i + o < 32 ? v[i + o] : v[i]);
        memcpy(v, w, sizeof(w));
    }
    return v[0];
}

/* sum of E over the real planes in the device's reduction order */
static double blocked_sum(const oracle_ts *t)
{
    const int gx = (t->ncells + TS_CELLS_PER_BLOCK - 1) / TS_CELLS_PER_BLOCK;
    const long np = (long)gx * t->nplanes;
    double *partial = (double *)malloc((size_t)np * sizeof(double));
    if (!partial) return NAN;
    double lane[TS_THREADS];
    for (int pl = 0; pl < t->nplanes; pl++) {
        const int col = t->plane_col[pl];
        for (int bx = 0; bx < gx; bx++) {
            int c0 = bx * TS_CELLS_PER_BLOCK;
            int c1 = c0 + TS_CELLS_PER_BLOCK < t->ncells ? c0 + TS_CELLS_PER_BLOCK : t->ncells;
            for (int i = 0; i < TS_THREADS; i++) lane[i] = 0.0;
            for (int i = 0; i < TS_THREADS; i++)
                for (int c = c0 + i; c < c1; c += TS_THREADS) lane[i] += t->E[(size_t)c * t->ndof + col];
            double tot = 0.0;
            for (int w = 0; w < TS_THREADS / 32; w++) tot += warp_tree(&lane[32 * w]);
            partial[(long)pl * gx + bx] = tot;
        }
    }
    double th[1024];
    for (int i = 0; i < 1024; i++) {
        th[i] = 0.0;
        for (long k = i; k < np; k += 1024) th[i] += partial[k];
    }
    double tot = 0.0;
    for (int w = 0; w < 32; w++) tot += warp_tree(&th[32 * w]);
    free(partial);
    return tot;
}

static double ts_dsp_next(oracle_ts *t, double h, double enorm, int accepted)
{
    const double k = (double)(t->eorder + 1);
    const double e = enorm > 1e-10 ? enorm : 1e-10;
    double r;
    if (accepted && t->have_prev) r = pow(e, -0.6 / k) * pow(t->e_prev, 0.2 / k);
    else r = pow(e, -1.0 / k);
    double rho = 1.0 + atan(r - 1.0);
    if (!accepted && rho > 0.9) rho = 0.9;
    if (accepted) { t->e_prev = e; t->have_prev = 1; }
    double dt = h * rho;
    return dt < t->o.dtmin ? t->o.dtmin : (dt > t->o.dtmax ? t->o.dtmax : dt);
}

/* out = X + sum_j w_j K_j over the real planes; AS copied */
static void lincomb(const oracle_ts *t, const double *X, int nk, const double *w, double *out)
{
    const size_t n = (size_t)t->ncells * t->ndof;
    memcpy(out, X, n * sizeof(double));
    for (int c = 0; c < t->ncells; c++)
        for (int pl = 0; pl < t->nplanes; pl++) {
            const size_t i = (size_t)c * t->ndof + t->plane_col[pl];
            double acc = 0.0;
            for (int j = 0; j < nk; j++) acc += w[j] * t->K[j][i];
            out[i] = X[i] + acc;
        }
}

int oracle_ts_step(oracle_ts *t, double *X, double t_end, int *accepted)
{
    const double t0 = t->st.t;
    double h = t->dt;
    int last = 0;
    if (t0 + h >= t_end) { h = t_end - t0; last = 1; }
    if (!(h > 0.0)) return 1;
    double w[TS_MAXSTAGES], we[TS_MAXSTAGES];
    for (int i = 0; i < t->ns; i++) {
        const double *Xi = X;
        if (i > 0) {
            for (int j = 0; j < i; j++) w[j] = h * t->A[i][j];
            lincomb(t, X, i, w, t->Y);
            Xi = t->Y;
        }
        int rc = oracle_rhs(t->p, t->m, t0 + t->c[i] * h, Xi, t->K[i]);
        if (rc) return rc;
        t->st.rhs_calls++;
    }
    for (int j = 0; j < t->ns; j++) { w[j] = h * t->b[j]; we[j] = h * t->bh[j]; }
    /* candidate, embedded solution and squared weighted errors */
    const size_t n = (size_t)t->ncells * t->ndof;
    memcpy(t->Y, X, n * sizeof(double));
    for (int c = 0; c < t->ncells; c++)
        for (int pl = 0; pl < t->nplanes; pl++) {
            const size_t i = (size_t)c * t->ndof + t->plane_col[pl];
            double acc = 0.0, acce = 0.0;
            for (int j = 0; j < t->ns; j++) {
                acc += w[j] * t->K[j][i];
                acce += we[j] * t->K[j][i];
            }
            const double xn = X[i] + acc, xe = X[i] + acce;
            t->Y[i] = xn;
            const double tol = t->o.abstol + t->o.reltol * fmax(fabs(xn), fabs(xe));
            const double e = (xn - xe) / tol;
            t->E[i] = e * e;
        }
    double enorm = 0.0;
    if (t->eorder) {
        const long N = (long)t->ncells * ((t->L.pf_size + 1) + t->L.pf_size + t->L.dp_size + t->L.ex_size + 1);
        enorm = sqrt(blocked_sum(t) / (double)N);
    }
    t->st.last_norm = enorm;
    int acc;
    if (!isfinite(enorm)) {
        acc = 0;
        if (t->dt <= t->o.dtmin) { t->st.rejected++; *accepted = 0; return 4; }
        double dt = t->dt * 0.1;
        t->dt = dt < t->o.dtmin ? t->o.dtmin : dt;
        t->st.rejected++;
    } else {
        acc = enorm <= 1.0 || h <= t->o.dtmin || !t->eorder;
        double dtn = t->eorder ? ts_dsp_next(t, h, enorm, acc) : t->dt;
        if (acc) {
            memcpy(X, t->Y, n * sizeof(double));
            t->st.t = last ? t_end : t0 + h;
            t->st.steps++;
            if (t->o.poststep) {
                int rc = oracle_poststep(t->p, t->m, X);
                if (rc) return rc;
            }
            if (!(last && h < t->dt)) t->dt = dtn;
        } else {
            t->st.rejected++;
            t->dt = dtn;
        }
    }
    t->st.dt = t->dt;
    *accepted = acc;
    return 0;
}

int oracle_ts_solve(oracle_ts *t, double *X, double t0, double t_end, cipher_ts_stats *stats)
{
    if (!(t_end > t0)) return 1;
    t->st.t = t0;
    const int64_t start = t->st.steps;
    while (t->st.t < t_end) {
        if (t->o.max_steps > 0 && t->st.steps - start >= t->o.max_steps) break;
        int acc = 0;
        int rc = oracle_ts_step(t, X, t_end, &acc);
        if (rc) { if (stats) *stats = t->st; return rc; }
    }
    if (stats) *stats = t->st;
    return 0;
}

void oracle_ts_get_stats(const oracle_ts *t, cipher_ts_stats *st) { *st = t->st; }
