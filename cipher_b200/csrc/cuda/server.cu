/*
 * server.cu - a request loop that serves many simulations on one GPU with
 * continuous batching (no counterpart in the reference, which runs one
 * simulation per job).
 *
 * Requests (a problem, an initial-state recipe, an end time) queue in
 * arrival order.  Each poll:
 *   1. admits queued requests in order while their device footprint (state,
 *      model tables, stepper buffers) fits the HBM budget and the active
 *      limit: builds the mesh, the context and the initial state on the
 *      device, and attaches the domain to the batch;
 *   2. takes one batched step of every admitted domain (cipher_batch_step:
 *      one graph launch, one synchronisation);
 *   3. retires finished or failed domains: copies the final state to host
 *      memory, frees the device memory, and records the timestamps.
 * A request's result is the one it gets when solved alone (the batch steps
 * each domain with its own control and arithmetic).
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <deque>
#include <new>
#include <vector>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "kernels.h"

using cipher::dev_alloc;
using cipher::dev_free;

int cipher_set_error(int code, const char *fmt, ...);

static double now_s()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

struct Request {
    int64_t id;
    cipher_problem *p;
    int kind;                      /* CIPHER_INIT_* */
    double width, t_end;
    int state;                     /* 0 queued, 1 active, 2 done */
    cipher_mesh *m;
    cipher_ctx *ctx;
    void *X;
    int slot;
    int64_t footprint;
    cipher_ts_stats st;
    int status, error;
    double t_submit, t_admit, t_finish;
    std::vector<double> result;    /* final state, reference AoS layout */
    int64_t ncells;
    int32_t ndof;
};

struct cipher_server {
    cipher_server_opts o;
    cipher_batch *batch;
    std::deque<int64_t> queue;
    std::vector<Request *> reqs;   /* by id */
    int64_t used, peak;
    int active;
    cipher_server_counters cnt;
    double *d_aos;                 /* reusable device buffer of results in AoS layout */
    size_t aos_cap;
};

static void drop_device(Request *r)
{
    /* pool frees do not wait: the request's work must be finished */
    cudaDeviceSynchronize();
    dev_free(r->X);
    r->X = nullptr;
    if (r->ctx) cipher_ctx_destroy(r->ctx);
    r->ctx = nullptr;
    if (r->m) cipher_mesh_free(r->m);
    r->m = nullptr;
}

extern "C" int cipher_server_create(const cipher_server_opts *o, cipher_server **out)
{
    if (!o || !out) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *out = NULL;
    if (o->hbm_budget <= 0 || o->max_active < 1) return cipher_set_error(CIPHER_E_ARG, "bad budget or active limit");
    cipher_server *s = new (std::nothrow) cipher_server();
    if (!s) return cipher_set_error(CIPHER_E_NOMEM, "host allocation");
    s->o = *o;
    int rc = cipher_batch_create(o->device, o->precision, &o->ts, &s->batch);
    if (rc) { delete s; return rc; }
    *out = s;
    return CIPHER_OK;
}

extern "C" void cipher_server_destroy(cipher_server *s)
{
    if (!s) return;
    for (Request *r : s->reqs) {
        if (!r) continue;
        if (r->state == 1) cipher_batch_detach(s->batch, r->slot);
        drop_device(r);
        cipher_problem_free(r->p);
        delete r;
    }
    cipher_batch_destroy(s->batch);
    cudaDeviceSynchronize();
    dev_free(s->d_aos);
    delete s;
}

extern "C" int cipher_server_submit(cipher_server *s, cipher_problem *p, int kind, double width, double t_end,
                                    int64_t *id)
{
    if (!s || !p || !id) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (kind != CIPHER_INIT_SHARP && kind != CIPHER_INIT_DIFFUSE) return cipher_set_error(CIPHER_E_ARG, "unknown initial state");
    if (!(t_end > 0.0)) return cipher_set_error(CIPHER_E_ARG, "t_end must be positive");
    Request *r = new (std::nothrow) Request();
    if (!r) return cipher_set_error(CIPHER_E_NOMEM, "host allocation");
    r->id = (int64_t)s->reqs.size();
    r->p = p;
    r->kind = kind;
    r->width = width;
    r->t_end = t_end;
    r->slot = -1;
    r->t_submit = now_s();
    s->reqs.push_back(r);
    s->queue.push_back(r->id);
    *id = r->id;
    return CIPHER_OK;
}

/* build the request's device domain; on failure the request is done with
 * that error (a request that can never run does not block the queue) */
static int admit(cipher_server *s, Request *r)
{
    /* a sharp start is built on the device from the voxel map and needs only
     * the grid; a diffuse start is built on the host over the full mesh */
    const int sharp = r->kind == CIPHER_INIT_SHARP;
    int rc = sharp ? cipher_mesh_grid(r->p, &r->m) : cipher_mesh_uniform(r->p, 0, r->p->resolution[r->p->dim - 1], &r->m);
    if (!rc) rc = cipher_ctx_create(r->p, r->m, s->o.precision, s->o.device, &r->ctx);
    cipher_state_layout L;
    if (!rc) rc = cipher_ctx_layout(r->ctx, &L);
    double *aos = nullptr, *d_aos = nullptr;
    if (!rc && sharp) {
        if (dev_alloc(&r->X, (size_t)L.bytes) != cudaSuccess) rc = CIPHER_E_NOMEM;
        if (!rc && cudaMemset(r->X, 0, (size_t)L.bytes) != cudaSuccess) rc = CIPHER_E_CUDA;
        if (!rc) rc = cipher_state_init_sharp(r->ctx, r->p->voxelphase, r->X, NULL);
        r->ncells = L.ncells;
        r->ndof = cipher_problem_aos_layout(r->p).ndof;
    } else if (!rc) {
        const cipher_aos_layout A = cipher_problem_aos_layout(r->p);
        const size_t nb = (size_t)r->m->ncells * A.ndof * sizeof(double);
        aos = (double *)malloc(nb);
        if (!aos) rc = CIPHER_E_NOMEM;
        if (!rc) rc = cipher_initial_state_diffuse_aos(r->p, r->m, r->width, aos);
        if (!rc && dev_alloc(&r->X, (size_t)L.bytes) != cudaSuccess) rc = CIPHER_E_NOMEM;
        if (!rc && cudaMemset(r->X, 0, (size_t)L.bytes) != cudaSuccess) rc = CIPHER_E_CUDA;
        if (!rc && dev_alloc(&d_aos, nb) != cudaSuccess) rc = CIPHER_E_NOMEM;
        if (!rc && cudaMemcpy(d_aos, aos, nb, cudaMemcpyHostToDevice) != cudaSuccess) rc = CIPHER_E_CUDA;
        if (!rc) rc = cipher_state_from_aos(r->ctx, d_aos, r->X, NULL);
        if (!rc) rc = cipher_chem_init(r->ctx, r->X, NULL);
        if (cudaDeviceSynchronize() != cudaSuccess && !rc) rc = CIPHER_E_CUDA;
        dev_free(d_aos);
        free(aos);
        r->ncells = r->m->ncells;
        r->ndof = A.ndof;
    }
    if (!rc) rc = cipher_batch_attach(s->batch, r->ctx, r->X, 0.0, r->t_end, &r->slot);
    r->t_admit = now_s();
    if (rc) {
        cudaGetLastError();
        drop_device(r);
        r->state = 2;
        r->status = CIPHER_BATCH_FAILED;
        r->error = rc;
        r->t_finish = r->t_admit;
        return rc;
    }
    r->state = 1;
    s->active++;
    return CIPHER_OK;
}

/* device bytes a request will hold: its state and context tables plus the
 * batch's stage buffers, estimated from the problem before anything is
 * allocated */
static int64_t footprint(const cipher_server *s, const cipher_problem *p)
{
    int64_t ncells = 1;
    for (int d = 0; d < p->dim; d++) ncells *= p->resolution[d];
    const int64_t stride = (ncells + 127) / 128 * 128;
    const int P = p->pf_size, S = p->maxsites * p->ndp;
    const int64_t rb = s->o.precision == CIPHER_PREC_FP64 ? 8 : 4;
    const int64_t state = stride * (2 * (P + 1) + rb * P + 8 * p->ndp + 8 * (int64_t)P * S + rb) + 5 * 256;
    const int64_t tables = (int64_t)p->npf * p->npf * 4 + (int64_t)p->nmat * (int64_t)sizeof(cipher_material) +
                           (int64_t)p->nf * 512 + stride * (2 * (P + 1) + 8 * (2 * p->ncp + 1));
    int ns = s->o.ts.scheme == CIPHER_TS_RK3BS ? 4 : s->o.ts.scheme == CIPHER_TS_RK2A ? 2 : 1;
    const int64_t stepper = (ns + 1) * state + stride * 2 * (P + 1) + ((ncells + 2047) / 2048) * (P + p->ndp + P * S + 1) * 8;
    return state + tables + stepper;
}

extern "C" int cipher_server_poll(cipher_server *s, int *queued, int *active, int *done)
{
    if (!s) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    s->cnt.polls++;
    double t0 = now_s();
    /* 1. admission in arrival order */
    while (!s->queue.empty() && s->active < s->o.max_active) {
        Request *r = s->reqs[s->queue.front()];
        const int64_t need = footprint(s, r->p);
        if (s->used + need > s->o.hbm_budget) {
            if (s->active == 0) {
                /* larger than the whole budget: it can never run */
                s->queue.pop_front();
                r->state = 2;
                r->status = CIPHER_BATCH_FAILED;
                r->error = CIPHER_E_NOMEM;
                r->t_admit = r->t_finish = now_s();
                continue;
            }
            break;
        }
        s->queue.pop_front();
        if (admit(s, r) == CIPHER_OK) {
            r->footprint = need;
            s->used += need;
            if (s->used > s->peak) s->peak = s->used;
        }
    }
    double t1 = now_s();
    s->cnt.t_admit += t1 - t0;
    /* 2. one step of every admitted domain */
    int running = 0;
    if (s->active > 0) {
        int rc = cipher_batch_step(s->batch, &running);
        if (rc) return rc;
        s->cnt.steps++;
        s->cnt.domain_steps += s->active;
    }
    double t2 = now_s();
    s->cnt.t_step += t2 - t1;
    /* 3. retirement */
    int ndone = 0;
    for (Request *r : s->reqs) {
        if (!r) continue;
        if (r->state == 1) {
            int status = 0, error = 0;
            cipher_batch_slot_stats(s->batch, r->slot, &r->st, &status, &error);
            if (status == CIPHER_BATCH_RUNNING) continue;
            int rc = cipher_batch_detach(s->batch, r->slot);
            r->status = status;
            r->error = error ? error : rc;
            r->result.resize((size_t)r->ncells * r->ndof);
            const size_t nb = r->result.size() * sizeof(double);
            if (nb > s->aos_cap) {
                cudaDeviceSynchronize();
                dev_free(s->d_aos);
                s->d_aos = nullptr;
                s->aos_cap = 0;
                if (dev_alloc(&s->d_aos, nb + nb / 2) == cudaSuccess) s->aos_cap = nb + nb / 2;
            }
            if (s->d_aos && cipher_state_to_aos(r->ctx, r->X, s->d_aos, NULL) == CIPHER_OK)
                cudaMemcpy(r->result.data(), s->d_aos, nb, cudaMemcpyDeviceToHost);
            drop_device(r);
            r->state = 2;
            r->t_finish = now_s();
            s->used -= r->footprint;
            s->active--;
        }
        if (r->state == 2) ndone++;
    }
    s->cnt.t_retire += now_s() - t2;
    if (queued) *queued = (int)s->queue.size();
    if (active) *active = s->active;
    if (done) *done = ndone;
    return CIPHER_OK;
}

extern "C" int cipher_server_get_counters(const cipher_server *s, cipher_server_counters *c)
{
    if (!s || !c) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *c = s->cnt;
    cipher_batch_get_counters(s->batch, &c->rebuilds, &c->graph_steps, &c->direct_steps);
    return CIPHER_OK;
}

extern "C" int cipher_server_result(const cipher_server *s, int64_t id, cipher_server_result_t *res, double *X)
{
    if (!s || !res || id < 0 || id >= (int64_t)s->reqs.size() || !s->reqs[id])
        return cipher_set_error(CIPHER_E_ARG, "no such request");
    const Request *r = s->reqs[id];
    memset(res, 0, sizeof(*res));
    res->state = r->state;
    res->status = r->status;
    res->error = r->error;
    res->stats = r->st;
    res->t_submit = r->t_submit;
    res->t_admit = r->t_admit;
    res->t_finish = r->t_finish;
    res->ncells = r->ncells;
    res->ndof = r->ndof;
    res->footprint = r->footprint;
    if (X && r->state == 2 && !r->result.empty()) memcpy(X, r->result.data(), r->result.size() * sizeof(double));
    return CIPHER_OK;
}

extern "C" int cipher_server_usage(const cipher_server *s, int64_t *used, int64_t *peak)
{
    if (!s) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (used) *used = s->used;
    if (peak) *peak = s->peak;
    return CIPHER_OK;
}

/* drop a finished request's host result and its problem */
extern "C" int cipher_server_release(cipher_server *s, int64_t id)
{
    if (!s || id < 0 || id >= (int64_t)s->reqs.size() || !s->reqs[id])
        return cipher_set_error(CIPHER_E_ARG, "no such request");
    Request *r = s->reqs[id];
    if (r->state != 2) return cipher_set_error(CIPHER_E_ARG, "request %lld has not finished", (long long)id);
    cipher_problem_free(r->p);
    delete r;
    s->reqs[id] = nullptr;
    return CIPHER_OK;
}
