/*
 * amr.cu - time stepping on an adapted mesh: the reference's main loop with
 * AMR (src/cipher.c:1365-1606 and 1607-1829).
 *
 * The forest starts at its finest level (the voxel grid of the problem).  The
 * SetUpProblem state (sets, phase fractions, temperature; chemistry from c0
 * on the device) is adapted `initcoarsen` times with the reference's marks
 * (refine where a leaf holds more than one phase, coarsen elsewhere:
 * src/cipher.c:1380-1386) and transferred on the host.  Then the state lives
 * on the device: the stepper takes `interval` accepted steps, the active
 * counts and sets come back to the host (2 bytes per slot and leaf), the
 * forest adapts, a context is built over the new mesh and the state moves to
 * it on the device (cipher_state_transfer); the step size carries over as
 * the reference's solparams.timestep does.
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "kernels.h"

int cipher_set_error(int code, const char *fmt, ...);

using cipher::dev_alloc;
using cipher::dev_free;

struct cipher_amr {
    const cipher_problem *p;
    cipher_amr_opts o;
    cipher_forest *f;
    cipher_mesh *m;
    cipher_ctx *ctx;
    cipher_ts *ts;
    void *X;
    cipher_state_layout lay;
    cipher_ts_stats st;          /* accumulated over adaptations */
    double t;
    int64_t adaptations;
};

static void amr_drop(cipher_amr *a)
{
    cudaDeviceSynchronize();
    if (a->ts) cipher_ts_destroy(a->ts);
    a->ts = nullptr;
    dev_free(a->X);
    a->X = nullptr;
    if (a->ctx) cipher_ctx_destroy(a->ctx);
    a->ctx = nullptr;
    if (a->m) cipher_mesh_free(a->m);
    a->m = nullptr;
}

/* context, state buffer and stepper over the forest's current mesh */
static int amr_build(cipher_amr *a, cipher_mesh *m, cipher_ctx **ctx, void **X, cipher_state_layout *lay)
{
    int rc = cipher_ctx_create(a->p, m, a->o.precision, a->o.device, ctx);
    if (rc) return rc;
    rc = cipher_ctx_layout(*ctx, lay);
    if (rc) return rc;
    if (dev_alloc(X, (size_t)lay->bytes) != cudaSuccess) return cipher_set_error(CIPHER_E_NOMEM, "AMR state");
    if (cudaMemset(*X, 0, (size_t)lay->bytes) != cudaSuccess) return cipher_set_error(CIPHER_E_CUDA, "AMR state");
    return CIPHER_OK;
}

extern "C" int cipher_amr_create(const cipher_problem *p, const cipher_amr_opts *o, cipher_amr **out)
{
    if (!p || !o || !out) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *out = nullptr;
    if (o->interval < 1 || o->initcoarsen < 0) return cipher_set_error(CIPHER_E_ARG, "interval >= 1, initcoarsen >= 0");
    cipher_amr *a = new (std::nothrow) cipher_amr();
    if (!a) return cipher_set_error(CIPHER_E_NOMEM, "host allocation");
    a->p = p;
    a->o = *o;
    a->o.ts.max_steps = o->interval;               /* one solve call per adaptation interval */
    int rc = cipher_forest_create(p->dim, o->nblocks, o->lmin, o->lmax, o->lmax, p->periodic, p->size, &a->f);
    int32_t fres[3];
    if (!rc) rc = cipher_forest_resolution(a->f, fres);
    for (int d = 0; !rc && d < p->dim; d++)
        if (fres[d] != p->resolution[d])
            rc = cipher_set_error(CIPHER_E_ARG, "forest grid %d differs from the voxel grid %d along %d", fres[d],
                                  p->resolution[d], d);
    /* the SetUpProblem state on the finest leaves, with its chemistry from
     * c0 computed on the device */
    cipher_mesh *m = nullptr;
    if (!rc) rc = cipher_forest_mesh(a->f, &m);
    const cipher_aos_layout A = cipher_problem_aos_layout(p);
    std::vector<double> X;
    if (!rc) {
        X.resize((size_t)m->ncells * A.ndof);
        rc = cipher_initial_state_aos(p, m, X.data());
    }
    if (!rc && p->ndp > 0) {
        cipher_ctx *c0 = nullptr;
        void *X0 = nullptr;
        cipher_state_layout L0;
        double *d_aos = nullptr;
        const size_t nb = X.size() * sizeof(double);
        rc = amr_build(a, m, &c0, &X0, &L0);
        if (!rc && dev_alloc(&d_aos, nb) != cudaSuccess) rc = cipher_set_error(CIPHER_E_NOMEM, "AMR setup");
        if (!rc && cudaMemcpy(d_aos, X.data(), nb, cudaMemcpyHostToDevice) != cudaSuccess) rc = CIPHER_E_CUDA;
        if (!rc) rc = cipher_state_from_aos(c0, d_aos, X0, nullptr);
        if (!rc) rc = cipher_chem_init(c0, X0, nullptr);
        if (!rc) rc = cipher_state_to_aos(c0, X0, d_aos, nullptr);
        if (!rc && cudaMemcpy(X.data(), d_aos, nb, cudaMemcpyDeviceToHost) != cudaSuccess) rc = CIPHER_E_CUDA;
        cudaDeviceSynchronize();
        dev_free(d_aos);
        dev_free(X0);
        if (c0) cipher_ctx_destroy(c0);
    }
    /* the initial adaptations (the reference's initcoarsen loop) */
    for (int it = 0; !rc && it < o->initcoarsen; it++) {
        std::vector<int8_t> mark((size_t)cipher_forest_nleaves(a->f));
        rc = cipher_forest_mark_active(a->f, X.data(), A.ndof, mark.data());
        if (!rc) rc = cipher_forest_adapt(a->f, mark.data(), X.data(), A.ndof, A.pf_offset);
        std::vector<double> Y;
        if (!rc) {
            Y.resize((size_t)cipher_forest_nleaves(a->f) * A.ndof);
            rc = cipher_forest_transfer_aos(a->f, X.data(), A.ndof, Y.data());
        }
        X.swap(Y);
    }
    if (m) cipher_mesh_free(m);
    m = nullptr;
    if (!rc) rc = cipher_forest_mesh(a->f, &a->m);
    if (!rc) rc = amr_build(a, a->m, &a->ctx, &a->X, &a->lay);
    if (!rc) {
        double *d_aos = nullptr;
        const size_t nb = X.size() * sizeof(double);
        if (dev_alloc(&d_aos, nb) != cudaSuccess) rc = cipher_set_error(CIPHER_E_NOMEM, "AMR setup");
        if (!rc && cudaMemcpy(d_aos, X.data(), nb, cudaMemcpyHostToDevice) != cudaSuccess) rc = CIPHER_E_CUDA;
        if (!rc) rc = cipher_state_from_aos(a->ctx, d_aos, a->X, nullptr);
        cudaDeviceSynchronize();
        dev_free(d_aos);
    }
    if (!rc) rc = cipher_ts_create(a->ctx, &a->o.ts, &a->ts);
    if (rc) {
        cipher_amr_destroy(a);
        return rc;
    }
    *out = a;
    return CIPHER_OK;
}

extern "C" void cipher_amr_destroy(cipher_amr *a)
{
    if (!a) return;
    amr_drop(a);
    cipher_forest_destroy(a->f);
    delete a;
}

/* adapt the forest by the device state's active sets and move the state */
static int amr_adapt(cipher_amr *a)
{
    const int P = a->lay.pf_size;
    const int64_t n = a->lay.ncells, S = a->lay.stride;
    /* the sets (count and ids) of every leaf: the marks and the family check */
    std::vector<uint16_t> as((size_t)(P + 1) * S);
    if (cudaMemcpy(as.data(), (const char *)a->X + a->lay.as_offset, as.size() * sizeof(uint16_t),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
        return cipher_set_error(CIPHER_E_CUDA, "AMR sets");
    std::vector<double> sets((size_t)n * (P + 1), 0.0);
    for (int64_t c = 0; c < n; c++) {
        const int cnt = as[c] <= P ? as[c] : P;
        sets[(size_t)c * (P + 1)] = (double)as[c];
        for (int k = 1; k <= cnt; k++) sets[(size_t)c * (P + 1) + k] = (double)as[(size_t)k * S + c];
    }
    std::vector<int8_t> mark((size_t)n);
    int rc = cipher_forest_mark_active(a->f, sets.data(), P + 1, mark.data());
    if (!rc) rc = cipher_forest_adapt(a->f, mark.data(), sets.data(), P + 1, P + 1);
    if (rc) return rc;
    const int64_t nn = cipher_forest_nleaves(a->f);
    std::vector<int64_t> s0((size_t)nn);
    std::vector<int32_t> ns((size_t)nn);
    rc = cipher_forest_transfer_plan(a->f, s0.data(), ns.data());
    cipher_mesh *m = nullptr;
    cipher_ctx *ctx = nullptr;
    void *X = nullptr;
    cipher_state_layout lay;
    if (!rc) rc = cipher_forest_mesh(a->f, &m);
    if (!rc) rc = amr_build(a, m, &ctx, &X, &lay);
    if (!rc) rc = cipher_state_transfer(ctx, X, a->ctx, a->X, s0.data(), ns.data(), nullptr);
    cipher_ts *ts = nullptr;
    if (!rc) rc = cipher_ts_create(ctx, &a->o.ts, &ts);
    if (!rc) rc = cipher_ts_set_dt(ts, a->st.dt);
    if (rc) {
        cudaDeviceSynchronize();
        if (ts) cipher_ts_destroy(ts);
        dev_free(X);
        if (ctx) cipher_ctx_destroy(ctx);
        if (m) cipher_mesh_free(m);
        return rc;
    }
    amr_drop(a);
    a->m = m;
    a->ctx = ctx;
    a->X = X;
    a->lay = lay;
    a->ts = ts;
    a->adaptations++;
    return CIPHER_OK;
}

extern "C" int cipher_amr_solve(cipher_amr *a, double t_end, int64_t max_steps, cipher_ts_stats *stats)
{
    if (!a) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    const int64_t start = a->st.steps;
    while (a->t < t_end && (max_steps <= 0 || a->st.steps - start < max_steps)) {
        cipher_ts_stats s;
        const cipher_ts_stats before = a->st;
        cipher_ts_stats tsb;
        cipher_ts_get_stats(a->ts, &tsb);
        int rc = cipher_ts_solve(a->ts, a->X, a->t, t_end, &s, nullptr);
        /* the stepper counts from its creation: add this call's share */
        a->st.steps = before.steps + (s.steps - tsb.steps);
        a->st.rejected = before.rejected + (s.rejected - tsb.rejected);
        a->st.rhs_calls = before.rhs_calls + (s.rhs_calls - tsb.rhs_calls);
        a->st.t = a->t = s.t;
        a->st.dt = s.dt;
        a->st.last_norm = s.last_norm;
        if (rc) {
            if (stats) *stats = a->st;
            return rc;
        }
        if (a->t < t_end && (s.steps - tsb.steps) >= a->o.interval) {
            rc = amr_adapt(a);
            if (rc) {
                if (stats) *stats = a->st;
                return rc;
            }
        }
    }
    if (stats) *stats = a->st;
    return CIPHER_OK;
}

extern "C" int cipher_amr_state(const cipher_amr *a, cipher_ctx **ctx, void **X, const cipher_mesh **m,
                                int64_t *adaptations)
{
    if (!a) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (ctx) *ctx = a->ctx;
    if (X) *X = a->X;
    if (m) *m = a->m;
    if (adaptations) *adaptations = a->adaptations;
    return CIPHER_OK;
}
