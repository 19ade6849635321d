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
#include <new>
#include <vector>
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
    int per_slot;                   /* planes per active-set slot (PF 1, EX S); 0: not slot planes */
};

struct CombineArgs {
    int64_t ncells, stride;
    int ngroups;
    PlaneGroup groups[4];
    int nk;
    const char *x;                  /* base state */
    const uint16_t *nact;           /* active counts of x (AS plane 0): slots at or past a cell's count are
                                       skipped; their derivatives are zero, so they change nothing and
                                       add exact zeros to the error sum */
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

/* the cells [c0, c1) of one plane (byte offset `off`) in element type E:
 * y = x + sum_j w_j k_j, and with NORM the thread's share of the weighted
 * error sum.  Stages are unrolled to kMaxStages (registers, no local
 * arrays); the operations and their order are those of the FP64 path. */
template <bool NORM, typename E>
__device__ __forceinline__ double combine_cells(const CombineArgs &a, int nk, const double *w, const double *we,
                                                int64_t off, int64_t c0, int64_t c1, int slot)
{
    const E *x = (const E *)(a.x + off);
    E *y = (E *)(a.y + off);
    const E *kp[kMaxStages];
#pragma unroll
    for (int j = 0; j < kMaxStages; j++) kp[j] = j < nk ? (const E *)(a.k[j] + off) : x;
    double sum = 0.0;
    for (int64_t c = c0 + threadIdx.x; c < c1; c += kTsThreads) {
        if (slot >= 0 && slot >= (int)__ldg(&a.nact[c])) continue;
        const double xv = (double)x[c];
        double acc = 0.0, acce = 0.0;
#pragma unroll
        for (int j = 0; j < kMaxStages; j++) {
            if (j < nk) {
                const double kv = (double)kp[j][c];
                acc += w[j] * kv;
                if (NORM) acce += we[j] * kv;
            }
        }
        const double xn = xv + acc;
        y[c] = (E)xn;
        if (NORM) {
            const double xe = xv + acce;
            const double tol = a.atol + a.rtol * fmax(fabs(xn), fabs(xe));
            const double e = (xn - xe) / tol;
            sum += e * e;
        }
    }
    return sum;
}

/* one block of a combination: cells [bx*2048, +2048) of state plane
 * `plane`; with NORM also the block's share of the weighted error sum,
 * written to *partial (the caller passes &partials[plane*gx + bx]) */
template <bool NORM>
__device__ __forceinline__ void rk_combine_block(const CombineArgs &a, int nk, const double *w, const double *we,
                                                 int plane, int64_t bx, double *partial)
{
    int gi = 0;
    while (gi < a.ngroups && plane >= a.groups[gi].nplanes) plane -= a.groups[gi++].nplanes;
    double sum = 0.0;
    if (gi < a.ngroups) {
        const PlaneGroup g = a.groups[gi];
        const int64_t off = g.offset + (int64_t)plane * a.stride * g.esize;
        const int64_t c0 = bx * kTsCellsPerBlock;
        const int64_t c1 = c0 + kTsCellsPerBlock < a.ncells ? c0 + kTsCellsPerBlock : a.ncells;
        const int slot = g.per_slot > 0 ? plane / g.per_slot : -1;
        sum = g.esize == 8 ? combine_cells<NORM, double>(a, nk, w, we, off, c0, c1, slot)
                           : combine_cells<NORM, float>(a, nk, w, we, off, c0, c1, slot);
    }
    if (NORM) {
        /* fixed-order block reduction: shuffle tree per warp, then the warps in order */
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        __shared__ double ws[kTsThreads / 32];
        if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int k = 0; k < kTsThreads / 32; k++) t += ws[k];
            partial[0] = t;
        }
    }
}

/* grid: x = cell blocks of kTsCellsPerBlock, y = plane over all groups */
template <bool NORM>
__global__ void __launch_bounds__(kTsThreads) k_rk_combine(const CombineArgs a)
{
    rk_combine_block<NORM>(a, a.nk, a.w, a.we, blockIdx.y, blockIdx.x,
                           a.partial + (int64_t)blockIdx.y * gridDim.x + blockIdx.x);
}

__device__ __forceinline__ void reduce_partials_block(const double *partial, int64_t n, double *out)
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

__global__ void __launch_bounds__(1024) k_reduce_partials(const double *partial, int64_t n, double *out)
{
    reduce_partials_block(partial, n, out);
}

/* ---------------- batched forms (one launch over many domains) ---------------- */

/* per-domain combination: the block list is the concatenation of every
 * domain's (plane, cell block) grid, plane-major as in the single form */
struct BatchCombine {
    const CombineArgs *args;      /* [n] device: x, y, k, groups, partial of each domain */
    const int64_t *tile_start;    /* [n+1]: domain i owns gx_i * nplanes_i blocks */
    const int64_t *gx;            /* [n] cell blocks per plane */
    const double *h;              /* [n] step size of each domain */
    const int *active;            /* [n] */
    int n;
    int64_t total;
    int nk;
    double coef[kMaxStages], coefe[kMaxStages];   /* tableau row (stage) or b / bhat (final) */
};

template <bool NORM>
__global__ void __launch_bounds__(kTsThreads) k_rk_combine_batched(const BatchCombine b)
{
    const int64_t t = blockIdx.x;
    int lo = 0, hi = b.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&b.tile_start[mid]) <= t) lo = mid;
        else hi = mid - 1;
    }
    if (!b.active[lo]) return;
    const CombineArgs &a = b.args[lo];
    const int64_t local = t - b.tile_start[lo], gx = b.gx[lo];
    const int plane = (int)(local / gx);
    const int64_t bx = local % gx;
    const double h = b.h[lo];
    double w[kMaxStages], we[kMaxStages];
#pragma unroll
    for (int j = 0; j < kMaxStages; j++) { w[j] = h * b.coef[j]; we[j] = h * b.coefe[j]; }
    rk_combine_block<NORM>(a, b.nk, w, we, plane, bx, a.partial + (int64_t)plane * gx + bx);
}

/* one block per domain: its partials reduced as the single form does */
__global__ void __launch_bounds__(1024) k_reduce_partials_batched(const CombineArgs *args, const int64_t *npartial,
                                                                  const int *active, double *out)
{
    const int i = blockIdx.x;
    if (!active[i]) return;
    reduce_partials_block(args[i].partial, npartial[i], &out[i]);
}

/* batched byte copies (16-byte units): domain i copies bytes[i] from src[i]
 * to dst[i] when flag[i] is set; blocks of 4096 units */
struct BatchCopy {
    const uint4 *const *src;
    uint4 *const *dst;
    const int64_t *units;         /* [n] */
    const int64_t *tile_start;    /* [n+1] */
    const int *flag;              /* [n] */
    int n;
    int64_t total;
};

__global__ void __launch_bounds__(256) k_copy_batched(const BatchCopy b)
{
    const int64_t t = blockIdx.x;
    int lo = 0, hi = b.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&b.tile_start[mid]) <= t) lo = mid;
        else hi = mid - 1;
    }
    if (!b.flag[lo]) return;
    const int64_t u0 = (t - b.tile_start[lo]) * 4096, n = b.units[lo];
    const uint4 *src = b.src[lo];
    uint4 *dst = b.dst[lo];
    for (int64_t u = u0 + threadIdx.x; u < u0 + 4096 && u < n; u += 256) dst[u] = src[u];
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
/* step control shared by the single and the batched stepper            */
/* ------------------------------------------------------------------ */

struct Control {
    double dt, e_prev;
    int have_prev;
    cipher_ts_stats st;
};

static double clamp_dt(const cipher_ts_opts &o, double dt)
{
    return dt < o.dtmin ? o.dtmin : (dt > o.dtmax ? o.dtmax : dt);
}

/* new step size from the normalised error (DSP filter PI.4.2 with the
 * smooth limiter); `accepted` selects whether e enters the filter history */
static double dsp_next(const Tableau &T, const cipher_ts_opts &o, Control &ct, double h, double enorm, int accepted)
{
    const double k = (double)(T.eorder + 1);
    const double e = enorm > 1e-10 ? enorm : 1e-10;
    double r;
    if (accepted && ct.have_prev) r = pow(e, -0.6 / k) * pow(ct.e_prev, 0.2 / k);
    else r = pow(e, -1.0 / k);
    double rho = 1.0 + atan(r - 1.0);
    if (!accepted && rho > 0.9) rho = 0.9;
    if (accepted) { ct.e_prev = e; ct.have_prev = 1; }
    return clamp_dt(o, h * rho);
}

/* step size of the next attempt from time st.t toward t_end */
static double attempt_h(const Control &ct, double t_end, int *last)
{
    double h = ct.dt;
    *last = 0;
    if (ct.st.t + h >= t_end) { h = t_end - ct.st.t; *last = 1; }
    return h;
}

/* accept or reject an attempt of size h with error norm enorm; updates the
 * controller and the statistics.  Returns 1 (accepted), 0 (rejected) or
 * -1 (non-finite norm at the minimum step: the domain has failed). */
static int decide(const Tableau &T, const cipher_ts_opts &o, Control &ct, double h, int last, double t_end,
                  double enorm)
{
    ct.st.last_norm = enorm;
    int acc;
    if (!std::isfinite(enorm)) {
        if (ct.dt <= o.dtmin) { ct.st.rejected++; return -1; }
        ct.dt = clamp_dt(o, ct.dt * 0.1);
        ct.st.rejected++;
        acc = 0;
    } else {
        acc = enorm <= 1.0 || h <= o.dtmin || !T.eorder;
        const double dtn = T.eorder ? dsp_next(T, o, ct, h, enorm, acc) : ct.dt;
        if (acc) {
            ct.st.t = last ? t_end : ct.st.t + h;
            ct.st.steps++;
            /* a shortened final step does not shrink the next one */
            if (!(last && h < ct.dt)) ct.dt = dtn;
        } else {
            ct.st.rejected++;
            ct.dt = dtn;
        }
    }
    ct.st.dt = ct.dt;
    return acc;
}

static int nplanes_of(const cipher_state_layout &L) { return L.pf_size + L.dp_size + L.ex_size + 1; }

static int64_t ndof_total_of(const cipher_state_layout &L)
{
    const int P = L.pf_size;
    return L.ncells * (int64_t)((P + 1) + P + L.dp_size + L.ex_size + 1);
}

static CombineArgs make_combine(const cipher_state_layout &L, const cipher_ts_opts &o, const void *X, void *Y,
                                void *const *K, int ns, double *partial)
{
    CombineArgs a;
    memset(&a, 0, sizeof(a));
    const int esize = L.precision == CIPHER_PREC_FP64 ? 8 : 4;
    a.ncells = L.ncells;
    a.stride = L.stride;
    int g = 0;
    a.groups[g++] = {L.pf_offset, L.pf_size, esize, 1};
    if (L.dp_size) a.groups[g++] = {L.dp_offset, L.dp_size, 8, 0};
    if (L.ex_size) a.groups[g++] = {L.ex_offset, L.ex_size, 8, L.ex_size / L.pf_size};
    a.groups[g++] = {L.tm_offset, 1, esize, 0};
    a.ngroups = g;
    a.x = (const char *)X;
    a.nact = (const uint16_t *)((const char *)X + L.as_offset);
    a.y = (char *)Y;
    for (int j = 0; j < ns; j++) a.k[j] = (const char *)K[j];
    a.atol = o.abstol;
    a.rtol = o.reltol;
    a.partial = partial;
    return a;
}

#define TS_CUDA(call, where)                                                                  \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return cipher_set_error(CIPHER_E_CUDA, "%s: %s", where, cudaGetErrorString(e_)); \
    } while (0)

static int check_opts(const cipher_ts_opts *o, Tableau *tab)
{
    if (!tableau(o->scheme, tab)) return cipher_set_error(CIPHER_E_ARG, "unknown RK scheme %d", o->scheme);
    if (!(o->dtmin > 0.0) || !(o->dtmax >= o->dtmin) || !(o->dt0 > 0.0))
        return cipher_set_error(CIPHER_E_ARG, "step limits must satisfy 0 < dtmin <= dtmax and dt0 > 0");
    if (tab->eorder && !(o->abstol > 0.0 || o->reltol > 0.0))
        return cipher_set_error(CIPHER_E_ARG, "tolerances must not both be zero");
    return CIPHER_OK;
}

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

/* ------------------------------------------------------------------ */
/* the stepper of one domain                                            */
/* ------------------------------------------------------------------ */

struct cipher_ts {
    cipher_ctx *ctx;
    cipher_ts_opts o;
    Tableau tab;
    cipher_state_layout lay;
    void *K[kMaxStages];
    void *Y;                       /* stage input and candidate solution */
    double *d_partial, *d_sum, *h_sum;
    int64_t npartial;
    Control ct;
    cipher_nucleation *nu;         /* nucleation before the active-set update, or NULL */
};

static dim3 combine_grid(const cipher_state_layout &L)
{
    return dim3((unsigned)((L.ncells + kTsCellsPerBlock - 1) / kTsCellsPerBlock), (unsigned)nplanes_of(L));
}

static void free_ts(cipher_ts *ts)
{
    if (!ts) return;
    /* pool frees do not wait: finish every queued use of the buffers first */
    cudaDeviceSynchronize();
    for (int j = 0; j < kMaxStages; j++) dev_free(ts->K[j]);
    dev_free(ts->Y);
    dev_free(ts->d_partial);
    dev_free(ts->d_sum);
    pinned_word_free(ts->h_sum);
    free(ts);
}

extern "C" int cipher_ts_create(cipher_ctx *c, const cipher_ts_opts *o, cipher_ts **out)
{
    if (!c || !o || !out) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *out = NULL;
    Tableau tab;
    int rc = check_opts(o, &tab);
    if (rc) return rc;
    cipher_ts *ts = (cipher_ts *)calloc(1, sizeof(cipher_ts));
    if (!ts) return cipher_set_error(CIPHER_E_NOMEM, "host allocation");
    ts->ctx = c;
    ts->o = *o;
    ts->tab = tab;
    rc = cipher_ctx_layout(c, &ts->lay);
    if (rc) { free(ts); return rc; }
    cudaError_t e = cudaSuccess;
    for (int j = 0; j < tab.ns && e == cudaSuccess; j++) e = dev_alloc(&ts->K[j], (size_t)ts->lay.bytes);
    if (e == cudaSuccess) e = dev_alloc(&ts->Y, (size_t)ts->lay.bytes);
    if (e == cudaSuccess) e = cudaMemset(ts->Y, 0, (size_t)ts->lay.bytes);
    dim3 g = combine_grid(ts->lay);
    ts->npartial = (int64_t)g.x * g.y;
    if (e == cudaSuccess) e = dev_alloc(&ts->d_partial, (size_t)ts->npartial * sizeof(double));
    if (e == cudaSuccess) e = dev_alloc(&ts->d_sum, sizeof(double));
    if (e == cudaSuccess) e = pinned_word_alloc(&ts->h_sum);
    if (e != cudaSuccess) {
        free_ts(ts);
        return cipher_set_error(CIPHER_E_NOMEM, "stepper buffers: %s", cudaGetErrorString(e));
    }
    ts->ct.dt = clamp_dt(*o, o->dt0);
    ts->ct.st.dt = ts->ct.dt;
    *out = ts;
    return CIPHER_OK;
}

extern "C" void cipher_ts_destroy(cipher_ts *ts) { free_ts(ts); }

extern "C" int cipher_ts_get_stats(const cipher_ts *ts, cipher_ts_stats *st)
{
    if (!ts || !st) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *st = ts->ct.st;
    return CIPHER_OK;
}

extern "C" int cipher_ts_set_dt(cipher_ts *ts, double dt)
{
    if (!ts || !(dt > 0.0)) return cipher_set_error(CIPHER_E_ARG, "dt must be positive");
    ts->ct.dt = clamp_dt(ts->o, dt);
    ts->ct.st.dt = ts->ct.dt;
    ts->ct.have_prev = 0;
    return CIPHER_OK;
}

/* one attempted step from X at time st.t, shortened to end at t_end */
extern "C" int cipher_ts_step(cipher_ts *ts, void *X, double t_end, int *accepted, void *stream)
{
    if (!ts || !X || !accepted) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    const Tableau &T = ts->tab;
    const double t = ts->ct.st.t;
    int last;
    const double h = attempt_h(ts->ct, t_end, &last);
    if (!(h > 0.0)) return cipher_set_error(CIPHER_E_ARG, "no time left before t_end");
    const cipher_state_layout &L = ts->lay;
    /* stage inputs share X's active sets (they change only in PostStep) */
    if (T.ns > 1)
        TS_CUDA(cudaMemcpyAsync((char *)ts->Y + L.as_offset, (const char *)X + L.as_offset,
                                (size_t)(L.pf_offset - L.as_offset), cudaMemcpyDeviceToDevice, s), "copy sets");
    dim3 grid = combine_grid(L);
    for (int i = 0; i < T.ns; i++) {
        const void *Xi = X;
        if (i > 0) {
            CombineArgs a = make_combine(L, ts->o, X, ts->Y, ts->K, i, nullptr);
            a.nk = i;
            for (int j = 0; j < i; j++) a.w[j] = h * T.A[i][j];
            k_rk_combine<false><<<grid, kTsThreads, 0, s>>>(a);
            TS_CUDA(cudaGetLastError(), "stage combine");
            Xi = ts->Y;
        }
        int rc = cipher_rhs(ts->ctx, t + T.c[i] * h, Xi, ts->K[i], stream);
        if (rc) return rc;
        ts->ct.st.rhs_calls++;
    }
    /* candidate solution, embedded solution and error sum in one pass */
    CombineArgs a = make_combine(L, ts->o, X, ts->Y, ts->K, T.ns, ts->d_partial);
    a.nk = T.ns;
    for (int j = 0; j < T.ns; j++) { a.w[j] = h * T.b[j]; a.we[j] = h * T.bh[j]; }
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
    const double enorm = T.eorder ? sqrt(*ts->h_sum / (double)ndof_total_of(L)) : 0.0;
    const int acc = decide(T, ts->o, ts->ct, h, last, t_end, enorm);
    *accepted = acc > 0;
    if (acc < 0) return cipher_set_error(CIPHER_E_NONFINITE, "non-finite error norm at the minimum step");
    if (acc) {
        /* the candidate becomes the solution */
        TS_CUDA(cudaMemcpyAsync((char *)X + L.pf_offset, (const char *)ts->Y + L.pf_offset,
                                (size_t)(L.bytes - L.pf_offset), cudaMemcpyDeviceToDevice, s), "accept");
        if (ts->nu) {
            int nfired = 0;
            rc = cipher_nucleation_step(ts->nu, X, ts->ct.st.t, h, &nfired, stream);
            if (rc) return rc;
            /* a nucleus restarts the step size from the minimum (src/cipher.c:861) */
            if (nfired) {
                ts->ct.dt = ts->o.dtmin;
                ts->ct.st.dt = ts->ct.dt;
                ts->ct.have_prev = 0;
            }
        }
        if (ts->o.poststep) {
            rc = cipher_poststep(ts->ctx, X, stream);
            if (rc) return rc;
        }
    }
    return CIPHER_OK;
}

extern "C" int cipher_ts_set_nucleation(cipher_ts *ts, struct cipher_nucleation *nu)
{
    if (!ts) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    ts->nu = nu;
    return CIPHER_OK;
}

extern "C" int cipher_ts_solve(cipher_ts *ts, void *X, double t0, double t_end, cipher_ts_stats *stats, void *stream)
{
    if (!ts || !X) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (!(t_end > t0)) return cipher_set_error(CIPHER_E_ARG, "t_end must exceed t0");
    ts->ct.st.t = t0;
    const int64_t start = ts->ct.st.steps;
    while (ts->ct.st.t < t_end) {
        if (ts->o.max_steps > 0 && ts->ct.st.steps - start >= ts->o.max_steps) break;
        int acc = 0;
        int rc = cipher_ts_step(ts, X, t_end, &acc, stream);
        if (rc) {
            if (stats) *stats = ts->ct.st;
            return rc;
        }
    }
    if (stats) *stats = ts->ct.st;
    return CIPHER_OK;
}

/* ------------------------------------------------------------------ */
/* many domains stepped together                                        */
/* ------------------------------------------------------------------ */
/*
 * Every attached domain takes one attempted step per cipher_batch_step with
 * its own step size and error control (the single stepper's control, so a
 * domain's trajectory is the one it has alone).  One step is one launch
 * sequence, captured once in a CUDA graph and replayed while the set of
 * domains is unchanged:
 *   H2D control block (step sizes, running flags, accept flags)
 *   accepted candidates of the previous step -> X, batched PostStep
 *   active sets X -> Y, then per stage: batched stage combination, the
 *   phase-field RHS of every kernel group in one persistent launch each,
 *   general-kernel domains one launch each
 *   batched final combination with per-domain error sums, per-domain norms
 *   D2H norms and error flags
 * followed by one host synchronisation.  Accepted candidates are moved into
 * X at the start of the next launch (or by cipher_batch_flush/detach), in
 * the same order of operations as the single stepper.
 */

struct BatchSlot {
    int used, status, error;       /* status: CIPHER_BATCH_* */
    cipher_ctx *ctx;
    void *X;
    CtxInfo info;
    cipher_state_layout lay;
    void *K[kMaxStages], *Y;
    uint16_t *pruned;
    double *partial;
    int64_t gx, npartial;
    Control ct;
    double t_end;
    int pending;                   /* accepted candidate not yet moved into X */
    int last;
    double h;
};

struct RhsGroup {
    int dim = 0, single = 0, pmax = 0, by = 2, grid = 0;
    int64_t maxstride = 0;
    std::vector<int> members;      /* dense indices */
    void *d_args[kMaxStages] = {}; /* PfArgs<R>[m] per stage */
    int64_t *d_tile_start = nullptr;
    int64_t total = 0;
    int goff = 0;                  /* offset of its running flags in the control block */
};

struct TuneKey {
    int precision, dim, single, pbucket, size_log2;
    int by, grid;
};

struct cipher_batch {
    int device, precision, nsm;
    cipher_ts_opts o;
    Tableau T;
    cudaStream_t stream;
    std::vector<BatchSlot> slots;
    std::vector<int> dense;        /* dense index -> slot */
    int dirty, use_graphs;
    /* device tables */
    std::vector<RhsGroup> groups;
    CombineArgs *d_comb;
    int64_t *d_comb_start, *d_gx, *d_npartial, comb_total;
    const uint4 **d_cp_src;
    uint4 **d_cp_dst;
    int64_t *d_cp_units, *d_cp_start, cp_total;          /* accept copies Y -> X */
    const uint4 **d_as_src;
    uint4 **d_as_dst;
    int64_t *d_as_units, *d_as_start, as_total;          /* active sets X -> Y */
    void *d_post;
    int64_t *d_post_start, post_total;
    int64_t *d_post_rows, post_row_total;
    int post_pmax;
    /* control block: double h[n] | int active[n] | int accept[n] | int gactive[sum m] */
    char *d_ctl, *h_ctl;
    size_t ctl_bytes;
    /* outputs: double norm[n] | int err[n] */
    char *d_out, *h_out;
    size_t out_bytes;
    cudaGraphExec_t graph;
    int stable_steps;             /* steps since the last rebuild */
    int64_t n_rebuilds, n_graph_steps, n_direct_steps;
    std::vector<TuneKey> tuned;
    /* launch tables live in one device arena, filled by one copy */
    char *d_arena;
    size_t arena_cap, ctl_cap, out_cap;
    std::vector<char> staging;
    std::vector<std::pair<void **, size_t>> fixups;
};


static double *ctl_h(char *base) { return (double *)base; }

/* append a table to the host staging area; its device pointer is set when
 * the arena is committed */
template <typename T_>
static void stage(cipher_batch *b, T_ **dptr, const std::vector<T_> &v)
{
    size_t off = (b->staging.size() + 255) / 256 * 256;
    b->staging.resize(off + v.size() * sizeof(T_));
    if (!v.empty()) memcpy(b->staging.data() + off, v.data(), v.size() * sizeof(T_));
    b->fixups.push_back({(void **)dptr, off});
}

static int commit_arena(cipher_batch *b)
{
    const size_t need = b->staging.size() + 256;
    if (need > b->arena_cap) {
        cudaDeviceSynchronize();
        dev_free(b->d_arena);
        b->d_arena = nullptr;
        b->arena_cap = 0;
        const size_t cap = need + need / 2;
        TS_CUDA(dev_alloc(&b->d_arena, cap), "batch tables");
        b->arena_cap = cap;
    }
    if (!b->staging.empty())
        TS_CUDA(cudaMemcpy(b->d_arena, b->staging.data(), b->staging.size(), cudaMemcpyHostToDevice), "batch tables");
    for (auto &f : b->fixups) *f.first = b->d_arena + f.second;
    b->staging.clear();
    b->fixups.clear();
    return CIPHER_OK;
}

/* grow-only device / pinned buffers of the control block and the outputs */
static int ensure_io(cipher_batch *b, size_t ctl, size_t out)
{
    if (ctl > b->ctl_cap) {
        cudaDeviceSynchronize();
        dev_free(b->d_ctl);
        if (b->h_ctl) cudaFreeHost(b->h_ctl);
        b->d_ctl = nullptr;
        b->h_ctl = nullptr;
        b->ctl_cap = 0;
        const size_t cap = ctl + ctl / 2 + 256;
        TS_CUDA(dev_alloc(&b->d_ctl, cap), "batch control");
        TS_CUDA(cudaMallocHost(&b->h_ctl, cap), "batch control");
        b->ctl_cap = cap;
    }
    if (out > b->out_cap) {
        cudaDeviceSynchronize();
        dev_free(b->d_out);
        if (b->h_out) cudaFreeHost(b->h_out);
        b->d_out = nullptr;
        b->h_out = nullptr;
        b->out_cap = 0;
        const size_t cap = out + out / 2 + 256;
        TS_CUDA(dev_alloc(&b->d_out, cap), "batch outputs");
        TS_CUDA(cudaMallocHost(&b->h_out, cap), "batch outputs");
        b->out_cap = cap;
    }
    return CIPHER_OK;
}

/* forget the launch tables (their memory is reused by the next rebuild) */
static void free_tables(cipher_batch *b)
{
    b->groups.clear();
    b->d_comb = nullptr;
    b->d_comb_start = b->d_gx = b->d_npartial = nullptr;
    b->d_cp_src = nullptr;
    b->d_cp_dst = nullptr;
    b->d_cp_units = b->d_cp_start = nullptr;
    b->d_as_src = nullptr;
    b->d_as_dst = nullptr;
    b->d_as_units = b->d_as_start = nullptr;
    b->d_post = nullptr;
    b->d_post_start = nullptr;
    b->d_post_rows = nullptr;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->stable_steps = 0;
}

static void free_buffers(cipher_batch *b)
{
    free_tables(b);
    cudaDeviceSynchronize();
    dev_free(b->d_arena);
    dev_free(b->d_ctl);
    dev_free(b->d_out);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->h_out) cudaFreeHost(b->h_out);
    b->d_arena = b->d_ctl = b->d_out = b->h_ctl = b->h_out = nullptr;
    b->arena_cap = b->ctl_cap = b->out_cap = 0;
}

static void free_slot(BatchSlot &s)
{
    cudaDeviceSynchronize();
    for (int j = 0; j < kMaxStages; j++) dev_free(s.K[j]);
    dev_free(s.Y);
    dev_free(s.pruned);
    dev_free(s.partial);
    memset(&s, 0, sizeof(s));
}

extern "C" int cipher_batch_create(int device, int precision, const cipher_ts_opts *o, cipher_batch **out)
{
    if (!o || !out) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    *out = NULL;
    if (precision != CIPHER_PREC_FP64 && precision != CIPHER_PREC_MIXED)
        return cipher_set_error(CIPHER_E_ARG, "unknown precision %d", precision);
    Tableau tab;
    int rc = check_opts(o, &tab);
    if (rc) return rc;
    TS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    cipher_batch *b = new (std::nothrow) cipher_batch();
    if (!b) return cipher_set_error(CIPHER_E_NOMEM, "host allocation");
    b->device = device;
    b->precision = precision;
    b->o = *o;
    b->T = tab;
    b->use_graphs = 1;
    b->dirty = 1;
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return cipher_set_error(CIPHER_E_CUDA, "stream creation failed");
    }
    *out = b;
    return CIPHER_OK;
}

extern "C" void cipher_batch_destroy(cipher_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    free_buffers(b);
    for (auto &s : b->slots)
        if (s.used) free_slot(s);
    cudaStreamDestroy(b->stream);
    delete b;
}

/* device bytes a domain of this context takes in a batch, beyond its state X */
extern "C" int cipher_batch_footprint(const cipher_batch *b, const cipher_ctx *c, int64_t *bytes)
{
    if (!b || !c || !bytes) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    cipher_state_layout L;
    int rc = cipher_ctx_layout(c, &L);
    if (rc) return rc;
    const int64_t gx = (L.ncells + kTsCellsPerBlock - 1) / kTsCellsPerBlock;
    *bytes = (int64_t)(b->T.ns + 1) * L.bytes + (int64_t)(L.pf_size + 1) * L.stride * 2 +
             gx * nplanes_of(L) * 8;
    return CIPHER_OK;
}

extern "C" int cipher_batch_attach(cipher_batch *b, cipher_ctx *c, void *X, double t0, double t_end, int *slot)
{
    if (!b || !c || !X || !slot) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (!(t_end > t0)) return cipher_set_error(CIPHER_E_ARG, "t_end must exceed t0");
    CtxInfo info = ctx_info(c);
    if (info.device != b->device || info.precision != b->precision)
        return cipher_set_error(CIPHER_E_ARG, "context device/precision differ from the batch's");
    for (auto &s : b->slots)
        if (s.used && s.info.dim != info.dim)
            return cipher_set_error(CIPHER_E_ARG, "all domains of a batch have the same dimension");
    TS_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
    BatchSlot s;
    memset(&s, 0, sizeof(s));
    s.used = 1;
    s.status = CIPHER_BATCH_RUNNING;
    s.ctx = c;
    s.X = X;
    s.info = info;
    int rc = cipher_ctx_layout(c, &s.lay);
    if (rc) return rc;
    s.gx = (s.lay.ncells + kTsCellsPerBlock - 1) / kTsCellsPerBlock;
    s.npartial = s.gx * nplanes_of(s.lay);
    cudaError_t e = cudaSuccess;
    for (int j = 0; j < b->T.ns && e == cudaSuccess; j++) e = dev_alloc(&s.K[j], (size_t)s.lay.bytes);
    if (e == cudaSuccess) e = dev_alloc(&s.Y, (size_t)s.lay.bytes);
    if (e == cudaSuccess) e = cudaMemset(s.Y, 0, (size_t)s.lay.bytes);
    if (e == cudaSuccess) e = dev_alloc(&s.pruned, (size_t)(s.lay.pf_size + 1) * s.lay.stride * sizeof(uint16_t));
    if (e == cudaSuccess) e = dev_alloc(&s.partial, (size_t)s.npartial * sizeof(double));
    if (e != cudaSuccess) {
        free_slot(s);
        cudaGetLastError();
        return cipher_set_error(CIPHER_E_NOMEM, "batch domain buffers: %s", cudaGetErrorString(e));
    }
    s.ct.dt = clamp_dt(b->o, b->o.dt0);
    s.ct.st.dt = s.ct.dt;
    s.ct.st.t = t0;
    s.t_end = t_end;
    int idx = -1;
    for (size_t i = 0; i < b->slots.size(); i++)
        if (!b->slots[i].used) { idx = (int)i; break; }
    if (idx < 0) { idx = (int)b->slots.size(); b->slots.push_back(s); }
    else b->slots[idx] = s;
    b->dirty = 1;
    *slot = idx;
    return CIPHER_OK;
}

/* move one domain's accepted candidate into X and update its active sets */
static int apply_pending(cipher_batch *b, BatchSlot &s)
{
    if (!s.pending) return CIPHER_OK;
    const cipher_state_layout &L = s.lay;
    TS_CUDA(cudaMemcpyAsync((char *)s.X + L.pf_offset, (const char *)s.Y + L.pf_offset,
                            (size_t)(L.bytes - L.pf_offset), cudaMemcpyDeviceToDevice, b->stream), "accept");
    s.pending = 0;
    if (b->o.poststep) return cipher_poststep(s.ctx, s.X, b->stream);
    TS_CUDA(cudaStreamSynchronize(b->stream), "sync");
    return CIPHER_OK;
}

extern "C" int cipher_batch_flush(cipher_batch *b)
{
    if (!b) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    TS_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
    for (auto &s : b->slots) {
        if (!s.used || !s.pending) continue;
        int rc = apply_pending(b, s);
        if (rc) { s.status = CIPHER_BATCH_FAILED; s.error = rc; return rc; }
    }
    return CIPHER_OK;
}

extern "C" int cipher_batch_detach(cipher_batch *b, int slot)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
        return cipher_set_error(CIPHER_E_ARG, "no such batch slot");
    TS_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
    BatchSlot &s = b->slots[slot];
    int rc = apply_pending(b, s);
    TS_CUDA(cudaStreamSynchronize(b->stream), "sync");
    free_slot(s);
    b->dirty = 1;
    return rc;
}

extern "C" int cipher_batch_slot_stats(const cipher_batch *b, int slot, cipher_ts_stats *st, int *status, int *error)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
        return cipher_set_error(CIPHER_E_ARG, "no such batch slot");
    const BatchSlot &s = b->slots[slot];
    if (st) *st = s.ct.st;
    if (status) *status = s.status;
    if (error) *error = s.error;
    return CIPHER_OK;
}

extern "C" int cipher_batch_set_graphs(cipher_batch *b, int on)
{
    if (!b) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    b->use_graphs = on ? 1 : 0;
    b->dirty = 1;
    return CIPHER_OK;
}

static int pbucket(int P) { return P <= 4 ? 4 : P <= 8 ? 8 : P <= 12 ? 12 : 16; }

/* BatchTiles tile prefix of a group for tile rows `by` */
static std::vector<int64_t> group_tiles(const cipher_batch *b, const RhsGroup &g, int by)
{
    std::vector<int64_t> st(g.members.size() + 1, 0);
    for (size_t k = 0; k < g.members.size(); k++) {
        const CtxInfo &in = b->slots[b->dense[g.members[k]]].info;
        const int64_t tx = (in.res[0] + 31) / 32, ty = (in.res[1] + by - 1) / by;
        st[k + 1] = st[k] + tx * ty * in.res[2];
    }
    return st;
}

template <typename R>
static BatchTiles<R> group_batch(const cipher_batch *b, const RhsGroup &g, int stage)
{
    BatchTiles<R> t;
    t.args = (const PfArgs<R> *)g.d_args[stage];
    t.tile_start = g.d_tile_start;
    t.active = (const int *)(b->d_ctl + g.goff);
    t.n = (int)g.members.size();
    t.total = g.total;
    t.pmax = g.pmax;
    {
        const int64_t planes = g.pmax > 2 * g.dim ? g.pmax : 2 * g.dim;
        t.i32 = planes * g.maxstride < ((int64_t)1 << 31) - 1;
    }
    return t;
}

static cudaError_t launch_group(const cipher_batch *b, const RhsGroup &g, int stage, int by, int grid)
{
    if (b->precision == CIPHER_PREC_FP64)
        return launch_rhs_pf_batched(group_batch<double>(b, g, stage), g.dim, g.single, by, grid, b->stream);
    return launch_rhs_pf_batched(group_batch<float>(b, g, stage), g.dim, g.single, by, grid, b->stream);
}

/* time the candidate tile shapes and persistent grid sizes of a group on
 * its own domains (stage-0 RHS into K_0, which every step overwrites) and
 * keep the fastest; results are cached per (precision, dim, interface
 * kind, P bucket, size class) */
static int set_group_shape(RhsGroup &g, const cipher_batch *b, int by, int grid)
{
    g.by = by;
    g.grid = grid;
    std::vector<int64_t> st = group_tiles(b, g, by);
    TS_CUDA(cudaMemcpy(g.d_tile_start, st.data(), st.size() * sizeof(int64_t), cudaMemcpyHostToDevice), "tiles");
    g.total = st.back();
    return CIPHER_OK;
}

static int autotune_group(cipher_batch *b, RhsGroup &g)
{
    int size_log2 = 0;
    for (int64_t v = group_tiles(b, g, 2).back(); v > 1; v >>= 1) size_log2++;
    for (const TuneKey &k : b->tuned)
        if (k.precision == b->precision && k.dim == g.dim && k.single == g.single && k.pbucket == pbucket(g.pmax) &&
            k.size_log2 == size_log2)
            return set_group_shape(g, b, k.by, k.grid);
    cudaEvent_t e0, e1;
    TS_CUDA(cudaEventCreate(&e0), "event");
    TS_CUDA(cudaEventCreate(&e1), "event");
    float best = 1e30f;
    int best_by = 2, best_grid = b->nsm * 4;
    const int bys[3] = {1, 2, 4}, mults[4] = {2, 4, 8, 16};
    for (int bi = 0; bi < 3; bi++) {
        std::vector<int64_t> st = group_tiles(b, g, bys[bi]);
        TS_CUDA(cudaMemcpy(g.d_tile_start, st.data(), st.size() * sizeof(int64_t), cudaMemcpyHostToDevice), "tiles");
        g.total = st.back();
        for (int mi = 0; mi < 4; mi++) {
            int64_t grid = (int64_t)b->nsm * mults[mi];
            if (grid > g.total) grid = g.total;
            if (grid < 1) grid = 1;
            TS_CUDA(launch_group(b, g, 0, bys[bi], (int)grid), "autotune launch");
            TS_CUDA(cudaEventRecord(e0, b->stream), "event");
            for (int r = 0; r < 3; r++) TS_CUDA(launch_group(b, g, 0, bys[bi], (int)grid), "autotune launch");
            TS_CUDA(cudaEventRecord(e1, b->stream), "event");
            TS_CUDA(cudaEventSynchronize(e1), "event");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) { best = ms; best_by = bys[bi]; best_grid = (int)grid; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc = set_group_shape(g, b, best_by, best_grid);
    if (rc) return rc;
    TuneKey k = {b->precision, g.dim, g.single, pbucket(g.pmax), size_log2, g.by, g.grid};
    b->tuned.push_back(k);
    /* the candidates wrote K_0 and may have raised flags on the domains'
     * error words: clear them */
    TS_CUDA(cudaMemsetAsync(b->d_out + sizeof(double) * b->dense.size(), 0, sizeof(int) * b->dense.size(), b->stream), "clear flags");
    TS_CUDA(cudaStreamSynchronize(b->stream), "sync");
    return CIPHER_OK;
}

static int rebuild(cipher_batch *b)
{
    b->n_rebuilds++;
    free_tables(b);
    b->dense.clear();
    for (size_t i = 0; i < b->slots.size(); i++)
        if (b->slots[i].used) b->dense.push_back((int)i);
    const int n = (int)b->dense.size();
    b->dirty = 0;
    if (n == 0) return CIPHER_OK;
    const int ns = b->T.ns;
    /* RHS groups: phase-field domains by (dim, interface kind); general ones alone */
    for (int i = 0; i < n; i++) {
        const BatchSlot &s = b->slots[b->dense[i]];
        if (s.info.general) continue;
        RhsGroup *g = nullptr;
        for (auto &q : b->groups)
            if (q.dim == s.info.dim && q.single == s.info.single) g = &q;
        if (!g) {
            RhsGroup q;
            q.dim = s.info.dim;
            q.single = s.info.single;
            b->groups.push_back(q);
            g = &b->groups.back();
        }
        g->members.push_back(i);
        if (s.info.P > g->pmax) g->pmax = s.info.P;
        if (s.lay.stride > g->maxstride) g->maxstride = s.lay.stride;
    }
    size_t gsum = 0;
    for (auto &g : b->groups) gsum += g.members.size();
    /* control block and outputs first: kernel arguments point into them */
    b->ctl_bytes = (size_t)n * sizeof(double) + (size_t)(2 * n + gsum) * sizeof(int);
    b->out_bytes = (size_t)n * (sizeof(double) + sizeof(int));
    int rc0 = ensure_io(b, b->ctl_bytes, b->out_bytes);
    if (rc0) return rc0;
    TS_CUDA(cudaMemset(b->d_ctl, 0, b->ctl_bytes), "batch control");
    memset(b->h_ctl, 0, b->ctl_bytes);
    TS_CUDA(cudaMemset(b->d_out, 0, b->out_bytes), "batch outputs");
    int *d_err = (int *)(b->d_out + sizeof(double) * n);
    size_t goff = (size_t)n * sizeof(double) + (size_t)2 * n * sizeof(int);
    for (auto &g : b->groups) {
        g.goff = (int)goff;
        goff += g.members.size() * sizeof(int);
        for (int stg = 0; stg < ns; stg++) {
            if (b->precision == CIPHER_PREC_FP64) {
                std::vector<PfArgs<double>> v;
                for (int i : g.members) {
                    BatchSlot &s = b->slots[b->dense[i]];
                    v.push_back(ctx_pf_args_d(s.ctx, stg == 0 ? s.X : s.Y, s.K[stg], d_err + i));
                }
                stage(b, (PfArgs<double> **)&g.d_args[stg], v);
            } else {
                std::vector<PfArgs<float>> v;
                for (int i : g.members) {
                    BatchSlot &s = b->slots[b->dense[i]];
                    v.push_back(ctx_pf_args_f(s.ctx, stg == 0 ? s.X : s.Y, s.K[stg], d_err + i));
                }
                stage(b, (PfArgs<float> **)&g.d_args[stg], v);
            }
        }
        stage(b, &g.d_tile_start, std::vector<int64_t>(g.members.size() + 1, 0));
    }
    /* combinations */
    {
        std::vector<CombineArgs> v;
        std::vector<int64_t> st(1, 0), gx, np;
        for (int i = 0; i < n; i++) {
            BatchSlot &s = b->slots[b->dense[i]];
            v.push_back(make_combine(s.lay, b->o, s.X, s.Y, s.K, ns, s.partial));
            st.push_back(st.back() + s.npartial);
            gx.push_back(s.gx);
            np.push_back(s.npartial);
        }
        b->comb_total = st.back();
        stage(b, &b->d_comb, v);
        stage(b, &b->d_comb_start, st);
        stage(b, &b->d_gx, gx);
        stage(b, &b->d_npartial, np);
    }
    /* copies */
    {
        std::vector<const uint4 *> cs, as;
        std::vector<uint4 *> cd, ad;
        std::vector<int64_t> cu, au, cst(1, 0), ast(1, 0);
        for (int i = 0; i < n; i++) {
            BatchSlot &s = b->slots[b->dense[i]];
            const cipher_state_layout &L = s.lay;
            cs.push_back((const uint4 *)((const char *)s.Y + L.pf_offset));
            cd.push_back((uint4 *)((char *)s.X + L.pf_offset));
            cu.push_back((L.bytes - L.pf_offset) / 16);
            cst.push_back(cst.back() + (cu.back() + 4095) / 4096);
            as.push_back((const uint4 *)((const char *)s.X + L.as_offset));
            ad.push_back((uint4 *)((char *)s.Y + L.as_offset));
            au.push_back((L.pf_offset - L.as_offset) / 16);
            ast.push_back(ast.back() + (au.back() + 4095) / 4096);
        }
        b->cp_total = cst.back();
        b->as_total = ast.back();
        stage(b, (const uint4 ***)&b->d_cp_src, cs);
        stage(b, &b->d_cp_dst, cd);
        stage(b, &b->d_cp_units, cu);
        stage(b, &b->d_cp_start, cst);
        stage(b, (const uint4 ***)&b->d_as_src, as);
        stage(b, &b->d_as_dst, ad);
        stage(b, &b->d_as_units, au);
        stage(b, &b->d_as_start, ast);
    }
    /* PostStep */
    {
        std::vector<int64_t> st(1, 0), rows(1, 0);
        int pmax = 1;
        for (int i = 0; i < n; i++) {
            const BatchSlot &sl = b->slots[b->dense[i]];
            st.push_back(st.back() + (sl.lay.ncells + 255) / 256);
            rows.push_back(rows.back() + post_row_blocks(sl.info.res));
            if (sl.lay.pf_size > pmax) pmax = sl.lay.pf_size;
        }
        b->post_total = st.back();
        b->post_row_total = rows.back();
        b->post_pmax = pmax;
        stage(b, &b->d_post_start, st);
        stage(b, &b->d_post_rows, rows);
        if (b->precision == CIPHER_PREC_FP64) {
            std::vector<PostArgs<double>> v;
            for (int i = 0; i < n; i++) {
                BatchSlot &s = b->slots[b->dense[i]];
                v.push_back(ctx_post_args_d(s.ctx, s.X, s.pruned, d_err + i));
            }
            stage(b, (PostArgs<double> **)&b->d_post, v);
        } else {
            std::vector<PostArgs<float>> v;
            for (int i = 0; i < n; i++) {
                BatchSlot &s = b->slots[b->dense[i]];
                v.push_back(ctx_post_args_f(s.ctx, s.X, s.pruned, d_err + i));
            }
            stage(b, (PostArgs<float> **)&b->d_post, v);
        }
    }
    {
        int rc = commit_arena(b);
        if (rc) return rc;
    }
    /* tile shapes: every group's domains run during tuning */
    {
        int *ga = (int *)(b->h_ctl + (size_t)n * sizeof(double) + (size_t)2 * n * sizeof(int));
        for (size_t k = 0; k < gsum; k++) ga[k] = 1;
        TS_CUDA(cudaMemcpy(b->d_ctl, b->h_ctl, b->ctl_bytes, cudaMemcpyHostToDevice), "control");
        for (auto &g : b->groups) {
            int rc = autotune_group(b, g);
            if (rc) return rc;
        }
    }
    return CIPHER_OK;
}

/* the launch sequence of one step (see the header of this section) */
static int launch_step(cipher_batch *b)
{
    const int n = (int)b->dense.size();
    const int ns = b->T.ns;
    cudaStream_t s = b->stream;
    const int *active = (const int *)(b->d_ctl + (size_t)n * sizeof(double));
    const int *accept = active + n;
    TS_CUDA(cudaMemsetAsync(b->d_out + sizeof(double) * n, 0, sizeof(int) * n, s), "clear flags");
    TS_CUDA(cudaMemcpyAsync(b->d_ctl, b->h_ctl, b->ctl_bytes, cudaMemcpyHostToDevice, s), "control");
    /* previous step's accepted candidates */
    {
        BatchCopy c = {b->d_cp_src, b->d_cp_dst, b->d_cp_units, b->d_cp_start, accept, n, b->cp_total};
        k_copy_batched<<<(unsigned)b->cp_total, 256, 0, s>>>(c);
        TS_CUDA(cudaGetLastError(), "accept copy");
        if (b->o.poststep) {
            const int dim = b->slots[b->dense[0]].info.dim;
            cudaError_t e;
            if (b->precision == CIPHER_PREC_FP64) {
                BatchPost<double> p = {(const PostArgs<double> *)b->d_post, b->d_post_start, accept, n, b->post_total,
                                       b->d_post_rows, b->post_row_total, b->post_pmax};
                e = launch_poststep_batched(p, dim, s);
            } else {
                BatchPost<float> p = {(const PostArgs<float> *)b->d_post, b->d_post_start, accept, n, b->post_total,
                                      b->d_post_rows, b->post_row_total, b->post_pmax};
                e = launch_poststep_batched(p, dim, s);
            }
            TS_CUDA(e, "batched poststep");
        }
    }
    /* this step */
    if (ns > 1) {
        BatchCopy c = {b->d_as_src, b->d_as_dst, b->d_as_units, b->d_as_start, active, n, b->as_total};
        k_copy_batched<<<(unsigned)b->as_total, 256, 0, s>>>(c);
        TS_CUDA(cudaGetLastError(), "set copy");
    }
    const double *h = (const double *)b->d_ctl;
    for (int i = 0; i < ns; i++) {
        if (i > 0) {
            BatchCombine c;
            memset(&c, 0, sizeof(c));
            c.args = b->d_comb; c.tile_start = b->d_comb_start; c.gx = b->d_gx; c.h = h; c.active = active;
            c.n = n; c.total = b->comb_total; c.nk = i;
            for (int j = 0; j < i; j++) c.coef[j] = b->T.A[i][j];
            k_rk_combine_batched<false><<<(unsigned)b->comb_total, kTsThreads, 0, s>>>(c);
            TS_CUDA(cudaGetLastError(), "stage combine");
        }
        for (auto &g : b->groups) TS_CUDA(launch_group(b, g, i, g.by, g.grid), "batched rhs");
        int *d_err = (int *)(b->d_out + sizeof(double) * n);
        for (int k = 0; k < n; k++) {
            BatchSlot &sl = b->slots[b->dense[k]];
            if (!sl.info.general) continue;
            TS_CUDA(ctx_rhs_general(sl.ctx, i == 0 ? sl.X : sl.Y, sl.K[i], d_err + k, s), "general rhs");
        }
    }
    {
        BatchCombine c;
        memset(&c, 0, sizeof(c));
        c.args = b->d_comb; c.tile_start = b->d_comb_start; c.gx = b->d_gx; c.h = h; c.active = active;
        c.n = n; c.total = b->comb_total; c.nk = ns;
        for (int j = 0; j < ns; j++) { c.coef[j] = b->T.b[j]; c.coefe[j] = b->T.bh[j]; }
        if (b->T.eorder) {
            k_rk_combine_batched<true><<<(unsigned)b->comb_total, kTsThreads, 0, s>>>(c);
            TS_CUDA(cudaGetLastError(), "final combine");
            k_reduce_partials_batched<<<n, 1024, 0, s>>>(b->d_comb, b->d_npartial, active, (double *)b->d_out);
            TS_CUDA(cudaGetLastError(), "norm reduce");
        } else {
            k_rk_combine_batched<false><<<(unsigned)b->comb_total, kTsThreads, 0, s>>>(c);
            TS_CUDA(cudaGetLastError(), "final combine");
        }
    }
    TS_CUDA(cudaMemcpyAsync(b->h_out, b->d_out, b->out_bytes, cudaMemcpyDeviceToHost, s), "outputs");
    return CIPHER_OK;
}

static int flag_error(int flags)
{
    if (flags & ERR_CAP) return CIPHER_E_CAP;
    if (flags & ERR_BADSET) return CIPHER_E_ARG;
    return CIPHER_E_NONFINITE;
}

extern "C" int cipher_batch_step(cipher_batch *b, int *running)
{
    if (!b) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    TS_CUDA(cudaSetDevice(b->device), "cudaSetDevice");
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    const int n = (int)b->dense.size();
    if (running) *running = 0;
    if (n == 0) return CIPHER_OK;
    double *h = ctl_h(b->h_ctl);
    int *active = (int *)(b->h_ctl + (size_t)n * sizeof(double));
    int *accept = active + n;
    int any = 0;
    for (int i = 0; i < n; i++) {
        BatchSlot &s = b->slots[b->dense[i]];
        accept[i] = s.pending;
        active[i] = s.status == CIPHER_BATCH_RUNNING;
        h[i] = 0.0;
        if (active[i]) {
            h[i] = attempt_h(s.ct, s.t_end, &s.last);
            s.h = h[i];
            any = 1;
        }
    }
    for (auto &g : b->groups) {
        int *ga = (int *)(b->h_ctl + g.goff);
        for (size_t k = 0; k < g.members.size(); k++) ga[k] = active[g.members[k]];
    }
    if (!any) return cipher_batch_flush(b);
    /* while the membership changes from step to step (a request loop
     * admitting and retiring), direct launches avoid re-instantiating a
     * graph per step; a graph is captured once it has held for 3 steps */
    b->stable_steps++;
    if (b->use_graphs && b->stable_steps > 3) {
        if (!b->graph) {
            cudaGraph_t gr;
            TS_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            int rc = launch_step(b);
            cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
            if (rc) return rc;
            TS_CUDA(e, "end capture");
            e = cudaGraphInstantiate(&b->graph, gr, 0);
            cudaGraphDestroy(gr);
            TS_CUDA(e, "graph instantiate");
        }
        TS_CUDA(cudaGraphLaunch(b->graph, b->stream), "graph launch");
        b->n_graph_steps++;
    } else {
        int rc = launch_step(b);
        if (rc) return rc;
        b->n_direct_steps++;
    }
    TS_CUDA(cudaStreamSynchronize(b->stream), "step sync");
    const double *norm = (const double *)b->h_out;
    const int *err = (const int *)(b->h_out + sizeof(double) * n);
    int nrun = 0;
    for (int i = 0; i < n; i++) {
        BatchSlot &s = b->slots[b->dense[i]];
        if (accept[i]) s.pending = 0;
        if (err[i] && s.status != CIPHER_BATCH_FAILED) {
            s.status = CIPHER_BATCH_FAILED;
            s.error = flag_error(err[i]);
            continue;
        }
        if (!active[i] || s.status != CIPHER_BATCH_RUNNING) continue;
        s.ct.st.rhs_calls += b->T.ns;
        const double enorm = b->T.eorder ? sqrt(norm[i] / (double)ndof_total_of(s.lay)) : 0.0;
        const int acc = decide(b->T, b->o, s.ct, s.h, s.last, s.t_end, enorm);
        if (acc < 0) { s.status = CIPHER_BATCH_FAILED; s.error = CIPHER_E_NONFINITE; continue; }
        if (acc) {
            s.pending = 1;
            if (s.ct.st.t >= s.t_end) s.status = CIPHER_BATCH_FINISHED;
        }
        if (s.status == CIPHER_BATCH_RUNNING) nrun++;
    }
    if (running) *running = nrun;
    return CIPHER_OK;
}

extern "C" int cipher_batch_get_counters(const cipher_batch *b, int64_t *rebuilds, int64_t *graph_steps,
                                         int64_t *direct_steps)
{
    if (!b) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (rebuilds) *rebuilds = b->n_rebuilds;
    if (graph_steps) *graph_steps = b->n_graph_steps;
    if (direct_steps) *direct_steps = b->n_direct_steps;
    return CIPHER_OK;
}
