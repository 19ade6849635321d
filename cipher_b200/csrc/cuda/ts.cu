/*
 * ts.cu - explicit Runge-Kutta time stepper with an embedded error estimate
 * and a DSP step-size controller, on device state vectors.  Replaces the
 * reference's PETSc TS set-up and time loop (InitializeTS, src/cipher.c:
 * 1097-1115: TSRK, TSADAPTDSP, step limits, tolerances; the loop at
 * 1589-1606 with TS_EXACTFINALTIME_MATCHSTEP and PostStep after every
 * accepted step).  PETSc is not available, so the tableaux, the error norm
 * and the controller are written from their published definitions:
 *
 *   tableaux  1fe  forward Euler (no error estimate: every step accepted)
 *             2a   Heun, order 2, embedded forward Euler (order 1)
 *             3bs  Bogacki-Shampine 3(2)
 *   norm      weighted RMS over all dofs of the reference layout,
 *             e_i = (x_i - xhat_i) / (atol + rtol*max(|x_i|, |xhat_i|)),
 *             ||e|| = sqrt(sum e_i^2 / N); AS entries count in N with e_i = 0
 *   control   Soderlind's digital filter PI.4.2 on the normalised error,
 *             rho = 1 + atan(r - 1) (smooth limiter), r = e^(-b1/k)
 *             e_prev^(-b2/k), b1 = 3/5, b2 = -1/5, k = embedded order + 1;
 *             a step is accepted when ||e|| <= 1 (or when dt is at dtmin);
 *             a non-finite norm rejects the step and cuts dt by 10
 *
 * Every vector operation is one kernel over the real planes of the state
 * (PF, DP, EX, TM, cells < ncells only); the final combination also forms
 * the embedded solution and the error sum in the same pass.  The error sum
 * is reduced in a fixed order (per-block partials, then one block), so a
 * trajectory is reproducible bit for bit from run to run.
 */
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "kernels.h"

using namespace cipher;

extern "C" const char *cipher_last_error(void);
int cipher_set_error(int code, const char *fmt, ...);

namespace cipher {

constexpr int kTsThreads = 256;
constexpr int kTsCellsPerBlock = 2048;
constexpr int kMaxStages = 4;

/* one plane group of the state: `nplanes` planes of `esize`-byte reals */
struct PlaneGroup {
    int64_t offset;
    int nplanes, esize;
};

struct CombineArgs {
    int64_t ncells, stride;
    int ngroups;
    PlaneGroup groups[4];
    int nk;
    const char *x;                  /* base state */
    const char *k[kMaxStages];      /* stage derivatives */
    double w[kMaxStages];           /* h * b_j (or h * a_ij) */
    double we[kMaxStages];          /* h * bhat_j (norm only) */
    char *y;                        /* output state (real planes only) */
    double atol, rtol;
    double *partial;                /* [gridDim.y * gridDim.x] when NORM */
};

__device__ __forceinline__ double load_real(const char *base, int esize, int64_t i)
{
    return esize == 8 ? ((const double *)base)[i] : (double)((const float *)base)[i];
}

__device__ __forceinline__ void store_real(char *base, int esize, int64_t i, double v)
{
    if (esize == 8) ((double *)base)[i] = v;
    else ((float *)base)[i] = (float)v;
}

/* grid: x = cell blocks of kTsCellsPerBlock, y = plane over all groups */
template <bool NORM>
__global__ void __launch_bounds__(kTsThreads) k_rk_combine(const CombineArgs a)
{
    int plane = blockIdx.y, gi = 0;
    while (gi < a.ngroups && plane >= a.groups[gi].nplanes) plane -= a.groups[gi++].nplanes;
    double sum = 0.0;
    if (gi < a.ngroups) {
        const PlaneGroup g = a.groups[gi];
        const int64_t off = g.offset + (int64_t)plane * a.stride * g.esize;
        const int64_t c0 = (int64_t)blockIdx.x * kTsCellsPerBlock;
        const int64_t c1 = c0 + kTsCellsPerBlock < a.ncells ? c0 + kTsCellsPerBlock : a.ncells;
        for (int64_t c = c0 + threadIdx.x; c < c1; c += kTsThreads) {
            const double x = load_real(a.x + off, g.esize, c);
            double acc = 0.0, acce = 0.0;
            for (int j = 0; j < a.nk; j++) {
                const double kv = load_real(a.k[j] + off, g.esize, c);
                acc += a.w[j] * kv;
                if (NORM) acce += a.we[j] * kv;
            }
            const double xn = x + acc;
            store_real(a.y + off, g.esize, c, xn);
            if (NORM) {
                const double xe = x + acce;
                const double tol = a.atol + a.rtol * fmax(fabs(xn), fabs(xe));
                const double e = (xn - xe) / tol;
                sum += e * e;
            }
        }
    }
    if (NORM) {
        /* fixed-order block reduction: shuffle tree per warp, then the warps in order */
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        __shared__ double ws[kTsThreads / 32];
        if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < kTsThreads / 32; w++) t += ws[w];
            a.partial[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
        }
    }
}

__global__ void __launch_bounds__(1024) k_reduce_partials(const double *partial, int64_t n, double *out)
{
    double sum = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += 1024) sum += partial[i];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 32; w++) t += ws[w];
        *out = t;
    }
}

}  // namespace cipher

/* ------------------------------------------------------------------ */
/* tableaux                                                             */
/* ------------------------------------------------------------------ */

struct Tableau {
    int ns, order, eorder;         /* stages, order, embedded order (0: none) */
    double A[kMaxStages][kMaxStages], b[kMaxStages], bh[kMaxStages], c[kMaxStages];
};

static int tableau(int scheme, Tableau *t)
{
    memset(t, 0, sizeof(*t));
    if (scheme == CIPHER_TS_RK1FE) {
        t->ns = 1; t->order = 1; t->eorder = 0;
        t->b[0] = 1.0;
    } else if (scheme == CIPHER_TS_RK2A) {
        t->ns = 2; t->order = 2; t->eorder = 1;
        t->A[1][0] = 1.0;
        t->b[0] = 0.5; t->b[1] = 0.5;
        t->bh[0] = 1.0; t->bh[1] = 0.0;
        t->c[1] = 1.0;
    } else if (scheme == CIPHER_TS_RK3BS) {
        t->ns = 4; t->order = 3; t->eorder = 2;
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

/* ------------------------------------------------------------------ */
/* the stepper                                                          */
/* ------------------------------------------------------------------ */

struct cipher_ts {
    cipher_ctx *ctx;
    cipher_ts_opts o;
    Tableau tab;
    cipher_state_layout lay;
    int64_t ndof_total;            /* N of the RMS norm: cells x reference dofs */
    int esize;
    void *K[kMaxStages];
    void *Y;                       /* stage input and candidate solution */
    double *d_partial, *d_sum, *h_sum;
    int64_t npartial;
    double dt, e_prev;
    int have_prev;
    cipher_ts_stats st;
};

static CombineArgs combine_args(const cipher_ts *ts, const void *X, void *Y)
{
    CombineArgs a;
    memset(&a, 0, sizeof(a));
    const cipher_state_layout &L = ts->lay;
    a.ncells = L.ncells;
    a.stride = L.stride;
    int g = 0;
    a.groups[g++] = {L.pf_offset, L.pf_size, ts->esize};
    if (L.dp_size) a.groups[g++] = {L.dp_offset, L.dp_size, 8};
    if (L.ex_size) a.groups[g++] = {L.ex_offset, L.ex_size, 8};
    a.groups[g++] = {L.tm_offset, 1, ts->esize};
    a.ngroups = g;
    a.x = (const char *)X;
    a.y = (char *)Y;
    a.atol = ts->o.abstol;
    a.rtol = ts->o.reltol;
    a.partial = ts->d_partial;
    return a;
}

static int nplanes_of(const cipher_state_layout &L) { return L.pf_size + L.dp_size + L.ex_size + 1; }

static dim3 combine_grid(const cipher_ts *ts)
{
    return dim3((unsigned)((ts->lay.ncells + kTsCellsPerBlock - 1) / kTsCellsPerBlock), (unsigned)nplanes_of(ts->lay));
}

#define TS_CUDA(call, where)                                                                  \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return cipher_set_error(CIPHER_E_CUDA, "%s: %s", where, cudaGetErrorString(e_)); \
    } while (0)

extern "C" int cipher_ts_default_opts(const cipher_problem *p, cipher_ts_opts *o)
{
    if (!p || !o) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    memset(o, 0, sizeof(*o));
    o->scheme = CIPHER_TS_RK2A;
    o->poststep = 1;
    o->dt0 = p->timestep0 > p->mintimestep ? p->timestep0 : p->mintimestep;
    o->dtmin = p->mintimestep;
    o->dtmax = p->maxtimestep;
    o->reltol = p->reltol;
    o->abstol = p->abstol;
    o->max_steps = 0;
    return CIPHER_OK;
}

static void free_ts(cipher_ts *ts)
{
    if (!ts) return;
    for (int j = 0; j < kMaxStages; j++) cudaFree(ts->K[j]);
    cudaFree(ts->Y);
    cudaFree(ts->d_partial);
    cudaFree(ts->d_sum);
    if (ts->h_sum) cudaFreeHost(ts->h_sum);
    free(ts);
}

extern "C" int cipher_ts_create(cipher_ctx *c, const cipher_ts_opts *o, cipher_ts **out)
{
    if (!c || !o || !out) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *out = NULL;
    Tableau tab;
    if (!tableau(o->scheme, &tab)) return cipher_set_error(CIPHER_E_ARG, "unknown RK scheme %d", o->scheme);
    if (!(o->dtmin > 0.0) || !(o->dtmax >= o->dtmin) || !(o->dt0 > 0.0))
        return cipher_set_error(CIPHER_E_ARG, "step limits must satisfy 0 < dtmin <= dtmax and dt0 > 0");
    if (tab.eorder && !(o->abstol > 0.0 || o->reltol > 0.0))
        return cipher_set_error(CIPHER_E_ARG, "tolerances must not both be zero");
    cipher_ts *ts = (cipher_ts *)calloc(1, sizeof(cipher_ts));
    if (!ts) return cipher_set_error(CIPHER_E_NOMEM, "host allocation");
    ts->ctx = c;
    ts->o = *o;
    ts->tab = tab;
    int rc = cipher_ctx_layout(c, &ts->lay);
    if (rc) { free(ts); return rc; }
    ts->esize = ts->lay.precision == CIPHER_PREC_FP64 ? 8 : 4;
    const int P = ts->lay.pf_size;
    ts->ndof_total = ts->lay.ncells * (int64_t)((P + 1) + P + ts->lay.dp_size + ts->lay.ex_size + 1);
    cudaError_t e = cudaSuccess;
    for (int j = 0; j < tab.ns && e == cudaSuccess; j++) e = cudaMalloc(&ts->K[j], (size_t)ts->lay.bytes);
    if (e == cudaSuccess) e = cudaMalloc(&ts->Y, (size_t)ts->lay.bytes);
    if (e == cudaSuccess) e = cudaMemset(ts->Y, 0, (size_t)ts->lay.bytes);
    dim3 g = combine_grid(ts);
    ts->npartial = (int64_t)g.x * g.y;
    if (e == cudaSuccess) e = cudaMalloc(&ts->d_partial, (size_t)ts->npartial * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ts->d_sum, sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&ts->h_sum, sizeof(double));
    if (e != cudaSuccess) {
        free_ts(ts);
        return cipher_set_error(CIPHER_E_NOMEM, "stepper buffers: %s", cudaGetErrorString(e));
    }
    ts->dt = o->dt0 < o->dtmin ? o->dtmin : (o->dt0 > o->dtmax ? o->dtmax : o->dt0);
    ts->st.dt = ts->dt;
    *out = ts;
    return CIPHER_OK;
}

extern "C" void cipher_ts_destroy(cipher_ts *ts) { free_ts(ts); }

extern "C" int cipher_ts_get_stats(const cipher_ts *ts, cipher_ts_stats *st)
{
    if (!ts || !st) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *st = ts->st;
    return CIPHER_OK;
}

extern "C" int cipher_ts_set_dt(cipher_ts *ts, double dt)
{
    if (!ts || !(dt > 0.0)) return cipher_set_error(CIPHER_E_ARG, "dt must be positive");
    ts->dt = dt < ts->o.dtmin ? ts->o.dtmin : (dt > ts->o.dtmax ? ts->o.dtmax : dt);
    ts->st.dt = ts->dt;
    ts->have_prev = 0;
    return CIPHER_OK;
}

/* new step size from the normalised error (DSP filter PI.4.2 with the
 * smooth limiter); `accepted` selects whether e enters the filter history */
static double dsp_next(cipher_ts *ts, double h, double enorm, int accepted)
{
    const double k = (double)(ts->tab.eorder + 1);
    const double e = enorm > 1e-10 ? enorm : 1e-10;
    double r;
    if (accepted && ts->have_prev) r = pow(e, -0.6 / k) * pow(ts->e_prev, 0.2 / k);
    else r = pow(e, -1.0 / k);
    double rho = 1.0 + atan(r - 1.0);
    if (!accepted && rho > 0.9) rho = 0.9;
    if (accepted) { ts->e_prev = e; ts->have_prev = 1; }
    double dt = h * rho;
    return dt < ts->o.dtmin ? ts->o.dtmin : (dt > ts->o.dtmax ? ts->o.dtmax : dt);
}

/* one attempted step from X at time st.t, shortened to end at t_end */
extern "C" int cipher_ts_step(cipher_ts *ts, void *X, double t_end, int *accepted, void *stream)
{
    if (!ts || !X) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    const Tableau &T = ts->tab;
    const double t = ts->st.t;
    double h = ts->dt;
    int last = 0;
    if (t + h >= t_end) { h = t_end - t; last = 1; }
    if (!(h > 0.0)) return cipher_set_error(CIPHER_E_ARG, "no time left before t_end");
    const cipher_state_layout &L = ts->lay;
    /* stage inputs share X's active sets (they change only in PostStep) */
    if (T.ns > 1)
        TS_CUDA(cudaMemcpyAsync((char *)ts->Y + L.as_offset, (const char *)X + L.as_offset,
                                (size_t)(L.pf_offset - L.as_offset), cudaMemcpyDeviceToDevice, s), "copy sets");
    dim3 grid = combine_grid(ts);
    for (int i = 0; i < T.ns; i++) {
        const void *Xi = X;
        if (i > 0) {
            CombineArgs a = combine_args(ts, X, ts->Y);
            a.nk = i;
            for (int j = 0; j < i; j++) { a.k[j] = (const char *)ts->K[j]; a.w[j] = h * T.A[i][j]; }
            k_rk_combine<false><<<grid, kTsThreads, 0, s>>>(a);
            TS_CUDA(cudaGetLastError(), "stage combine");
            Xi = ts->Y;
        }
        int rc = cipher_rhs(ts->ctx, t + T.c[i] * h, Xi, ts->K[i], stream);
        if (rc) return rc;
        ts->st.rhs_calls++;
    }
    /* candidate solution, embedded solution and error sum in one pass */
    CombineArgs a = combine_args(ts, X, ts->Y);
    a.nk = T.ns;
    for (int j = 0; j < T.ns; j++) { a.k[j] = (const char *)ts->K[j]; a.w[j] = h * T.b[j]; a.we[j] = h * T.bh[j]; }
    double enorm = 0.0;
    if (T.eorder) {
        k_rk_combine<true><<<grid, kTsThreads, 0, s>>>(a);
        TS_CUDA(cudaGetLastError(), "final combine");
        k_reduce_partials<<<1, 1024, 0, s>>>(ts->d_partial, ts->npartial, ts->d_sum);
        TS_CUDA(cudaGetLastError(), "norm reduce");
        TS_CUDA(cudaMemcpyAsync(ts->h_sum, ts->d_sum, sizeof(double), cudaMemcpyDeviceToHost, s), "read norm");
    } else {
        k_rk_combine<false><<<grid, kTsThreads, 0, s>>>(a);
        TS_CUDA(cudaGetLastError(), "final combine");
    }
    TS_CUDA(cudaStreamSynchronize(s), "step sync");
    int rc = cipher_ctx_check(ts->ctx, stream);
    if (rc) return rc;
    if (T.eorder) enorm = sqrt(*ts->h_sum / (double)ts->ndof_total);
    ts->st.last_norm = enorm;
    int acc;
    if (!std::isfinite(enorm)) {
        acc = 0;
        double dt = ts->dt * 0.1;
        if (ts->dt <= ts->o.dtmin) {
            ts->st.rejected++;
            *accepted = 0;
            return cipher_set_error(CIPHER_E_NONFINITE, "non-finite error norm at the minimum step");
        }
        ts->dt = dt < ts->o.dtmin ? ts->o.dtmin : dt;
    } else {
        acc = enorm <= 1.0 || h <= ts->o.dtmin || !T.eorder;
        double dtn = T.eorder ? dsp_next(ts, h, enorm, acc) : ts->dt;
        if (acc) {
            /* the candidate becomes the solution */
            TS_CUDA(cudaMemcpyAsync((char *)X + L.pf_offset, (const char *)ts->Y + L.pf_offset,
                                    (size_t)(L.bytes - L.pf_offset), cudaMemcpyDeviceToDevice, s), "accept");
            ts->st.t = last ? t_end : t + h;
            ts->st.steps++;
            if (ts->o.poststep) {
                rc = cipher_poststep(ts->ctx, X, stream);
                if (rc) return rc;
            }
            /* a shortened final step does not shrink the next one */
            if (!(last && h < ts->dt)) ts->dt = dtn;
        } else {
            ts->st.rejected++;
            ts->dt = dtn;
        }
    }
    ts->st.dt = ts->dt;
    *accepted = acc;
    return CIPHER_OK;
}

extern "C" int cipher_ts_solve(cipher_ts *ts, void *X, double t0, double t_end, cipher_ts_stats *stats, void *stream)
{
    if (!ts || !X) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (!(t_end > t0)) return cipher_set_error(CIPHER_E_ARG, "t_end must exceed t0");
    ts->st.t = t0;
    const int64_t start = ts->st.steps;
    while (ts->st.t < t_end) {
        if (ts->o.max_steps > 0 && ts->st.steps - start >= ts->o.max_steps) break;
        int acc = 0;
        int rc = cipher_ts_step(ts, X, t_end, &acc, stream);
        if (rc) {
            if (stats) *stats = ts->st;
            return rc;
        }
    }
    if (stats) *stats = ts->st;
    return CIPHER_OK;
}
