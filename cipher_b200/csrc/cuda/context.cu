/*
 * context.cu - device context and the C ABI entry points of include/cipher_b200.h.
 *
 * A context owns the device copies of the model tables and the scratch the
 * per-step update needs; state vectors X and F are owned by the caller (the
 * time stepper), as PETSc's TS owns X and F for the reference's RHSFunction
 * (src/cipher.c:27, 1107).
 */
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "kernels.h"
#include "models.cuh"
#include "general_common.cuh"

using namespace cipher;

/* ------------------------------------------------------------------ */
/* errors                                                               */
/* ------------------------------------------------------------------ */

static thread_local char g_errmsg[512] = "";

static int set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_errmsg, sizeof(g_errmsg), fmt, ap);
    va_end(ap);
    return code;
}

/* the same, for the other units of the library */
int cipher_set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_errmsg, sizeof(g_errmsg), fmt, ap);
    va_end(ap);
    return code;
}

/* the same, for the library's C host units (the message is already formatted) */
extern "C" int cipher_host_set_error(int code, const char *msg)
{
    snprintf(g_errmsg, sizeof(g_errmsg), "%s", msg);
    return code;
}

static int cuda_fail(cudaError_t e, const char *where)
{
    return set_error(CIPHER_E_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define CUDA_TRY(call, where)                              \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, where); \
    } while (0)

extern "C" const char *cipher_strerror(int code)
{
    switch (code) {
    case CIPHER_OK: return "ok";
    case CIPHER_E_ARG: return "invalid argument";
    case CIPHER_E_NOMEM: return "out of memory";
    case CIPHER_E_CAP: return "active-set superset exceeds the phase cap";
    case CIPHER_E_NONFINITE: return "non-finite value";
    case CIPHER_E_CUDA: return "CUDA error";
    case CIPHER_E_TIMEOUT: return "bounded device wait ran out";
    case CIPHER_E_UNSUPPORTED: return "configuration not supported on the device";
    case CIPHER_E_STEP: return "time step below the minimum";
    default: return "unknown error";
    }
}

extern "C" const char *cipher_last_error(void) { return g_errmsg; }

/* ------------------------------------------------------------------ */
/* context                                                              */
/* ------------------------------------------------------------------ */

struct cipher_ctx {
    int device, precision, dim;
    int res[3], per[3];
    int64_t ncells, stride;
    int P, npf, ncp, ndp, S, nmat;
    cipher_state_layout lay;
    cipher_aos_layout aos;
    int general;                  /* 1: chemistry / heat / boundary kernels (rhs_general.cu) */
    int aniso;                    /* gradient-based anisotropy: gradients of phi before the RHS */
    double cw[3];                 /* cell width per axis (centroids of the gradient weights) */
    double *d_grad;               /* [dim][P][stride] gradients (aniso) */
    int32_t *d_order, *d_order_cursor; /* cell grouping: order, class totals */
    int32_t *d_order_counts;      /* [kOrderClasses][blocks of 256 cells] */
    int nclass;
    uint32_t single_models;       /* GenArgs::single_models */
    /* (cell, phase) items of the cells of several phases (rhs_items.cu) */
    double *d_iscr;
    int32_t *d_ibase, *d_icell, *d_icount;
    int64_t icap;                 /* 0: no item path */
    int item_model;               /* GenArgs::item_model */
    int single;
    double sig0, mob0, wid0, tj0, ffactor, vol, junctionpenalty, delta;
    int has_temp_rate;
    double temp_rate;
    int interp, nbcs;
    DevBC bcs[CIPHER_MAXBC];
    /* an adapted (non-uniform) mesh: per-cell face lists, face factors and
     * cell volumes on the device (FaceLists); 0 on uniform grids */
    int listed;
    int rhs_form;                 /* CIPHER_RHS_*: FP64 single-interface kernel choice */
    int32_t *d_fl_start, *d_fl_nbr, *d_fl_face, *d_fl_bstart, *d_fl_blabel;
    double *d_fl_ff, *d_fl_vol, *d_fl_delta;
    int32_t *d_itflist;
    DevInterface *d_itfs;
    cipher_material *d_mat;
    double *d_t0;                 /* [npf] temperature0 of each phase's material */
    cipher_material *d_mat_spec;  /* the materials specialised at one temperature */
    MatV *d_matv;                 /* their CALPHAD tables evaluated (NULL: off) */
    double *d_tspec;
    int32_t *d_pmm;
    double *d_comp, *d_mob, *d_tcond;
    uint16_t *d_pruned;
    int *d_err;
    int *h_err;
    /* buffers of the host-AoS entry point, allocated on first use */
    double *d_aos_x, *d_aos_f;
    void *d_X, *d_F;
    /* its slab pipeline: copy-in, compute and copy-out streams and their
     * events, created on first use */
    int pipe_ready;
    cudaStream_t s_up, s_cp, s_dn;
    cudaEvent_t ev_start, ev_end, ev_up[32], ev_done[32];
};

static constexpr int kAosSlabs = 32;

static int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

/* problems the general kernels take: everything the reference's RHS does
 * except random sources (which call rand() inside the RHS) */
static int problem_supported(const cipher_problem *p, char *why, size_t len)
{
    if (p->gradient_calculation < 0 || p->gradient_calculation > 1) { snprintf(why, len, "gradient_calculation is 0 or 1"); return 0; }
    if (p->ncp < 1 || p->ncp > CIPHER_MAXCP || p->ndp != p->ncp - 1) { snprintf(why, len, "bad component count"); return 0; }
    if (p->nbcs < 0 || p->nbcs > CIPHER_MAXBC) { snprintf(why, len, "bad boundary condition count"); return 0; }
    for (int m = 0; m < p->nmat; m++) {
        const cipher_material *mat = &p->material[m];
        if (mat->model < CIPHER_CHEM_QUADRATIC || mat->model > CIPHER_CHEM_NONE) { snprintf(why, len, "material %d: unknown model", m); return 0; }
        if (p->ndp == 0 && mat->model != CIPHER_CHEM_NONE) { snprintf(why, len, "material %d: chemical model needs ncp > 1", m); return 0; }
        if (p->ndp == 0 && (mat->tconductivity.n || mat->specific_heat.n || mat->latent_heat.n)) {
            snprintf(why, len, "material %d: thermal model without chemistry reads an unset temperature in the reference", m);
            return 0;
        }
        if (mat->model == CIPHER_CHEM_CALPHAD2SL && p->maxsites < 2) { snprintf(why, len, "material %d: two sublattices need maxsites 2", m); return 0; }
        for (int s = 0; s < mat->nsources; s++)
            if (mat->sources[s].model != CIPHER_SOURCE_SINK) { snprintf(why, len, "material %d: random sources are not reproducible", m); return 0; }
    }
    for (int i = 0; i < p->nf; i++)
        for (int s = 0; s < p->interface[i].nsources; s++)
            if (p->interface[i].sources[s].model != CIPHER_SOURCE_SINK) { snprintf(why, len, "interface %d: random sources are not reproducible", i); return 0; }
    if (p->interpolation != CIPHER_INTERP_CUBIC && p->interpolation != CIPHER_INTERP_QUADRATIC &&
        p->interpolation != CIPHER_INTERP_LINEAR) { snprintf(why, len, "unknown interpolation"); return 0; }
    return 1;
}

/* gradient-based anisotropy changes results only where an interface has
 * anisotropy values (src/cipher.c:427-460) */
static int has_anisotropy(const cipher_problem *p)
{
    if (!p->gradient_calculation) return 0;
    for (int i = 0; i < p->nf; i++)
        if (p->interface[i].energy_naniso > 0 || p->interface[i].mobility_naniso > 0) return 1;
    return 0;
}

/* problems the phase-field-only kernels take: no chemistry, no heat, no
 * boundary faces, no reference energies (grain growth) */
static int phasefield_only(const cipher_problem *p)
{
    if (p->ndp != 0 || p->nbcs != 0) return 0;
    if (p->interpolation == CIPHER_INTERP_LINEAR) return 0;
    for (int m = 0; m < p->nmat; m++) {
        const cipher_material *mat = &p->material[m];
        if (mat->model != CIPHER_CHEM_NONE || mat->ref.n != 0 || mat->ref.logcoeff != 0.0) return 0;
        if (mat->tconductivity.n || mat->specific_heat.n || mat->latent_heat.n || mat->nsources) return 0;
    }
    for (int i = 0; i < p->nf; i++)
        if (p->interface[i].has_potential || p->interface[i].nsources) return 0;
    return 1;
}

static void free_ctx(cipher_ctx *c)
{
    if (!c) return;
    /* pool frees do not wait: finish every queued use of the buffers first */
    cudaDeviceSynchronize();
    dev_free(c->d_fl_start);
    dev_free(c->d_fl_nbr);
    dev_free(c->d_fl_face);
    dev_free(c->d_fl_bstart);
    dev_free(c->d_fl_blabel);
    dev_free(c->d_fl_ff);
    dev_free(c->d_fl_vol);
    dev_free(c->d_fl_delta);
    dev_free(c->d_itflist);
    dev_free(c->d_itfs);
    dev_free(c->d_mat);
    dev_free(c->d_t0);
    dev_free(c->d_mat_spec);
    dev_free(c->d_matv);
    dev_free(c->d_tspec);
    dev_free(c->d_pmm);
    dev_free(c->d_comp);
    dev_free(c->d_mob);
    dev_free(c->d_tcond);
    dev_free(c->d_pruned);
    dev_free(c->d_grad);
    dev_free(c->d_order);
    dev_free(c->d_order_cursor);
    dev_free(c->d_order_counts);
    dev_free(c->d_iscr);
    dev_free(c->d_ibase);
    dev_free(c->d_icell);
    dev_free(c->d_icount);
    dev_free(c->d_err);
    pinned_word_free(c->h_err);
    dev_free(c->d_aos_x);
    dev_free(c->d_aos_f);
    dev_free(c->d_X);
    dev_free(c->d_F);
    if (c->pipe_ready) {
        cudaStreamDestroy(c->s_up);
        cudaStreamDestroy(c->s_cp);
        cudaStreamDestroy(c->s_dn);
        cudaEventDestroy(c->ev_start);
        cudaEventDestroy(c->ev_end);
        for (int i = 0; i < kAosSlabs; i++) {
            cudaEventDestroy(c->ev_up[i]);
            cudaEventDestroy(c->ev_done[i]);
        }
    }
    free(c);
}

/* per-cell face lists of an adapted mesh (FaceLists): every face in the
 * mesh's face order is appended to its L and R cells' lists, so each list is
 * in the reference's face order; face factors and volumes exactly as the
 * reference forms them (src/cipher.c:273-275, FastPow src/utility.c:112-124) */
static double fast_pow(double base, unsigned e)
{
    double r = 1.0;
    while (e) {
        if (e & 1u) r *= base;
        e >>= 1;
        base *= base;
    }
    return r;
}

static int upload_face_lists(cipher_ctx *c, const cipher_mesh *m, int dim)
{
    const int64_t n = m->ncells, nf = m->nfaces, nbf = m->nbfaces;
    std::vector<int32_t> start(n + 1, 0), nbr(2 * nf), face(2 * nf), bstart(n + 1, 0), blabel(nbf > 0 ? nbf : 1);
    std::vector<double> ff(nf > 0 ? nf : 1), vol(n), delta(n);
    for (int64_t i = 0; i < n; i++) {
        delta[i] = m->cellgeom[i];
        vol[i] = fast_pow(m->cellgeom[i], (unsigned)dim);
    }
    for (int64_t f = 0; f < nf; f++) {
        const int32_t L = m->face_cells[2 * f], R = m->face_cells[2 * f + 1];
        if (L < 0 || L >= n || R < 0 || R >= n || L == R) return set_error(CIPHER_E_ARG, "face %lld has bad cells", (long long)f);
        start[L + 1]++;
        start[R + 1]++;
        const double dl = delta[L], dr = delta[R];
        ff[f] = 2.0 * (dl < dr ? vol[L] / dl : vol[R] / dr) / (dl + dr);
    }
    for (int64_t i = 0; i < n; i++) start[i + 1] += start[i];
    std::vector<int32_t> fill(start.begin(), start.end() - 1);
    for (int64_t f = 0; f < nf; f++) {
        const int32_t L = m->face_cells[2 * f], R = m->face_cells[2 * f + 1];
        nbr[fill[L]] = R | FACE_SELF_L;
        face[fill[L]++] = (int32_t)f;
        nbr[fill[R]] = L;
        face[fill[R]++] = (int32_t)f;
    }
    for (int64_t b = 0; b < nbf; b++) {
        const int32_t cell = m->bface_cell[b];
        if (cell < 0 || cell >= n) return set_error(CIPHER_E_ARG, "boundary face %lld has a bad cell", (long long)b);
        bstart[cell + 1]++;
    }
    for (int64_t i = 0; i < n; i++) bstart[i + 1] += bstart[i];
    std::vector<int32_t> bfill(bstart.begin(), bstart.end() - 1);
    for (int64_t b = 0; b < nbf; b++) blabel[bfill[m->bface_cell[b]]++] = m->bface_label[b];
    cudaError_t e = cudaSuccess;
    auto up = [&](auto **dst, const auto &v) {
        const size_t bytes = v.size() * sizeof(v[0]);
        if (e == cudaSuccess) e = dev_alloc(dst, bytes);
        if (e == cudaSuccess) e = cudaMemcpy(*dst, v.data(), bytes, cudaMemcpyHostToDevice);
    };
    up(&c->d_fl_start, start);
    up(&c->d_fl_nbr, nbr.size() ? nbr : std::vector<int32_t>(1, 0));
    up(&c->d_fl_face, face.size() ? face : std::vector<int32_t>(1, 0));
    up(&c->d_fl_bstart, bstart);
    up(&c->d_fl_blabel, blabel);
    up(&c->d_fl_ff, ff);
    up(&c->d_fl_vol, vol);
    up(&c->d_fl_delta, delta);
    if (e != cudaSuccess) return cuda_fail(e, "face lists");
    return CIPHER_OK;
}

static FaceLists face_lists(const cipher_ctx *c)
{
    FaceLists f;
    memset(&f, 0, sizeof(f));
    if (!c->listed) return f;
    f.start = c->d_fl_start;
    f.nbr = c->d_fl_nbr;
    f.face = c->d_fl_face;
    f.ff = c->d_fl_ff;
    f.vol = c->d_fl_vol;
    f.delta = c->d_fl_delta;
    f.bstart = c->d_fl_bstart;
    f.blabel = c->d_fl_blabel;
    return f;
}

extern "C" int cipher_ctx_create(const cipher_problem *p, const cipher_mesh *m, int precision, int device,
                                 cipher_ctx **out)
{
    if (!out) return set_error(CIPHER_E_ARG, "out is NULL");
    *out = NULL;
    if (!p || !m) return set_error(CIPHER_E_ARG, "problem or mesh is NULL");
    if (precision != CIPHER_PREC_FP64 && precision != CIPHER_PREC_MIXED)
        return set_error(CIPHER_E_ARG, "unknown precision %d", precision);
    if (m->ncells != m->nowned)
        return set_error(CIPHER_E_UNSUPPORTED, "device path needs a whole-domain mesh (no ghost cells)");
    if (!m->uniform && (!m->face_cells && m->nfaces > 0))
        return set_error(CIPHER_E_ARG, "an adapted mesh needs its face list");
    if (p->pf_size < 1 || p->pf_size > CIPHER_MAXAP) return set_error(CIPHER_E_ARG, "bad phase cap %d", p->pf_size);
    /* kernels launch one block row per (y, z) grid line */
    if ((p->dim > 1 && m->res[1] > 65535) || (p->dim > 2 && m->res[2] > 65535))
        return set_error(CIPHER_E_UNSUPPORTED, "grid lines above 65535 in y or z");
    /* kernels index cells with 32-bit integers */
    if ((int64_t)m->ncells > 2147483647LL - 1024)
        return set_error(CIPHER_E_UNSUPPORTED, "more than 2^31 cells on one context");
    char why[256];
    if (!problem_supported(p, why, sizeof(why))) return set_error(CIPHER_E_UNSUPPORTED, "%s", why);
    for (int a = 0; a < p->npf; a++)
        if (p->phasematerialmapping[a] < 0 || p->phasematerialmapping[a] >= p->nmat)
            return set_error(CIPHER_E_ARG, "phase %d maps to material %d", a, p->phasematerialmapping[a]);

    CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    cipher_ctx *c = (cipher_ctx *)calloc(1, sizeof(cipher_ctx));
    if (!c) return set_error(CIPHER_E_NOMEM, "host allocation");
    c->device = device;
    c->precision = precision;
    c->dim = p->dim;
    for (int d = 0; d < 3; d++) {
        c->res[d] = d < p->dim ? m->res[d] : 1;
        c->per[d] = d < p->dim ? (m->periodic[d] && m->res[d] > 1) : 0;
    }
    c->ncells = m->ncells;
    c->stride = align_up(c->ncells, 128);
    c->P = p->pf_size;
    c->npf = p->npf;
    c->ncp = p->ncp;
    c->ndp = p->ndp;
    c->S = p->maxsites * p->ndp;
    c->nmat = p->nmat;
    c->junctionpenalty = p->junctionpenalty;
    c->listed = !m->uniform;
    c->aniso = has_anisotropy(p);
    if (c->aniso && (c->listed || m->nowned != m->ncells)) {
        free_ctx(c);
        return set_error(CIPHER_E_UNSUPPORTED, "gradient-based anisotropy needs a whole-domain uniform grid");
    }
    for (int d = 0; d < 3; d++) c->cw[d] = d < p->dim ? p->size[d] / p->resolution[d] : 1.0;
    /* the phase-field kernels walk uniform grids; adapted meshes and
     * anisotropy take the general kernels */
    c->general = c->listed || !phasefield_only(p) || c->aniso;
    c->interp = p->interpolation;
    c->delta = m->cellgeom[0];
    c->nbcs = p->nbcs;
    for (int b = 0; b < p->nbcs; b++) {
        const cipher_bc *bc = &p->bcs[b];
        DevBC &d = c->bcs[b];
        d.label = bc->boundaryid;
        d.chem_type = bc->chem_bctype;
        d.thermal_type = bc->thermal_bctype;
        d.thermal_val = bc->thermal_bcval;
        for (int k = 0; k < CIPHER_MAXCP; k++) { d.chem_val[k] = bc->chem_bcval[k]; d.chem_on[k] = bc->chem_bcbool[k]; }
    }
    c->has_temp_rate = p->has_temperature_rate;
    c->temp_rate = p->has_temperature_rate ? p->temperature_rate[p->currentloadcase] : 0.0;
    c->aos = cipher_problem_aos_layout(p);

    /* geometry exactly as the reference forms it (src/cipher.c:273-275) */
    {
        double delta = m->cellgeom[0];
        double vol = 1.0, b = delta;
        unsigned e = (unsigned)p->dim;
        while (e) { if (e & 1u) vol *= b; e >>= 1; b *= b; }
        c->vol = vol;
        c->ffactor = 2.0 * (delta < delta ? vol / delta : vol / delta) / (delta + delta);
    }

    /* state layout */
    const int64_t rb = precision == CIPHER_PREC_FP64 ? 8 : 4;
    cipher_state_layout L;
    memset(&L, 0, sizeof(L));
    L.ncells = c->ncells;
    L.stride = c->stride;
    L.pf_size = c->P;
    L.dp_size = c->ndp;
    L.ex_size = c->P * c->S;
    L.precision = precision;
    int64_t off = 0;
    L.as_offset = off; off = align_up(off + (int64_t)(c->P + 1) * c->stride * 2, 256);
    /* face maps: one 32-bit word per slot (uniform grids only) */
    L.map_offset = off; L.map_planes = c->listed ? 0 : c->P;
    off = align_up(off + (int64_t)L.map_planes * c->stride * 4, 256);
    L.pf_offset = off; off = align_up(off + (int64_t)c->P * c->stride * rb, 256);
    L.dp_offset = off; off = align_up(off + (int64_t)c->ndp * c->stride * 8, 256);
    L.ex_offset = off; off = align_up(off + (int64_t)L.ex_size * c->stride * 8, 256);
    L.tm_offset = off; off = align_up(off + c->stride * rb, 256);
    L.bytes = off;
    c->lay = L;

    /* interface tables: one T-independent interface for every pair is the
     * common case (grain growth) and needs no lookup */
    int first = -1, single = 1;
    for (int a = 0; a < p->npf && single; a++)
        for (int b = a + 1; b < p->npf; b++) {
            int i = p->interfacelist[a * p->npf + b];
            if (i < 0 || i >= p->nf) { free_ctx(c); return set_error(CIPHER_E_ARG, "interface index %d out of range", i); }
            if (first < 0) first = i;
            else if (i != first) { single = 0; break; }
        }
    if (first < 0) first = 0;
    if (p->interface[first].energy_activation.n || p->interface[first].mobility_activation.n) single = 0;
    c->single = single;
    {
        const cipher_interface *itf = &p->interface[first];
        c->sig0 = 1.0 * itf->energy_m0;
        c->mob0 = 1.0 * itf->mobility_m0;
        c->wid0 = itf->width;
        double v = c->sig0 / c->wid0, t = 0.0;
        t = t > v ? t : v;
        t = t > v ? t : v;
        t = t > v ? t : v;
        t *= p->junctionpenalty;
        c->tj0 = t;
    }
    cudaError_t e;
    {   /* the pair table: the general kernels look pairs up; so does the output */
        for (int a = 0; a < p->npf; a++)
            for (int b = a + 1; b < p->npf; b++) {
                int i = p->interfacelist[a * p->npf + b];
                if (i < 0 || i >= p->nf) { free_ctx(c); return set_error(CIPHER_E_ARG, "interface index out of range"); }
            }
        size_t nb = (size_t)p->npf * p->npf * sizeof(int32_t);
        if ((e = dev_alloc(&c->d_itflist, nb)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc itflist"); }
        if ((e = cudaMemcpy(c->d_itflist, p->interfacelist, nb, cudaMemcpyHostToDevice)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "copy itflist"); }
    }
    {
        DevInterface *h = (DevInterface *)calloc((size_t)p->nf, sizeof(DevInterface));
        if (!h) { free_ctx(c); return set_error(CIPHER_E_NOMEM, "host allocation"); }
        for (int i = 0; i < p->nf; i++) {
            const cipher_interface *s = &p->interface[i];
            h[i].width = s->width;
            h[i].energy_m0 = s->energy_m0;
            h[i].mobility_m0 = s->mobility_m0;
            h[i].energy_act = s->energy_activation;
            h[i].mobility_act = s->mobility_activation;
            h[i].has_potential = s->has_potential;
            h[i].has_mobilityc = s->has_mobilityc;
            memcpy(h[i].potential, s->potential, sizeof(h[i].potential));
            memcpy(h[i].mobilityc, s->mobilityc, sizeof(h[i].mobilityc));
            h[i].nsources = s->nsources;
            memcpy(h[i].sources, s->sources, sizeof(h[i].sources));
            /* anisotropy acts only with gradient_calculation (src/cipher.c:427) */
            h[i].energy_n = p->gradient_calculation ? s->energy_naniso : 0;
            h[i].mobility_n = p->gradient_calculation ? s->mobility_naniso : 0;
            memcpy(h[i].energy_dir, s->energy_aniso_dir, sizeof(h[i].energy_dir));
            memcpy(h[i].energy_val, s->energy_aniso_val, sizeof(h[i].energy_val));
            memcpy(h[i].mobility_dir, s->mobility_aniso_dir, sizeof(h[i].mobility_dir));
            memcpy(h[i].mobility_val, s->mobility_aniso_val, sizeof(h[i].mobility_val));
        }
        e = dev_alloc(&c->d_itfs, (size_t)p->nf * sizeof(DevInterface));
        if (e == cudaSuccess) e = cudaMemcpy(c->d_itfs, h, (size_t)p->nf * sizeof(DevInterface), cudaMemcpyHostToDevice);
        free(h);
        if (e != cudaSuccess) { free_ctx(c); return cuda_fail(e, "interface table"); }
    }
    {
        size_t nb = (size_t)p->npf * sizeof(int32_t);
        if ((e = dev_alloc(&c->d_pmm, nb)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc phase map"); }
        if ((e = cudaMemcpy(c->d_pmm, p->phasematerialmapping, nb, cudaMemcpyHostToDevice)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "copy phase map"); }
    }
    if (c->general) {
        size_t nb = (size_t)p->nmat * sizeof(cipher_material);
        if ((e = dev_alloc(&c->d_mat, nb)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc materials"); }
        if ((e = cudaMemcpy(c->d_mat, p->material, nb, cudaMemcpyHostToDevice)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "copy materials"); }
        if ((e = dev_alloc(&c->d_mat_spec, nb)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc materials"); }
        /* [0] the copies' temperature, [1 + m] material m's copy, [1 + nmat + m] its evaluated tables */
        if ((e = dev_alloc(&c->d_tspec, (size_t)(1 + 2 * p->nmat) * sizeof(double))) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc materials"); }
        const char *senv = getenv("CIPHER_B200_SPECIALISED_KERNELS");
        if ((!senv || strcmp(senv, "0") != 0) &&
            (e = dev_alloc(&c->d_matv, (size_t)p->nmat * sizeof(MatV))) != cudaSuccess) {
            free_ctx(c);
            return cuda_fail(e, "cudaMalloc evaluated materials");
        }
        {
            std::vector<double> nan((size_t)(1 + 2 * p->nmat), std::nan(""));
            if ((e = cudaMemcpy(c->d_tspec, nan.data(), nan.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "copy"); }
        }
        if (c->ndp) {
            nb = (size_t)c->ncp * c->stride * sizeof(double);
            if ((e = dev_alloc(&c->d_comp, nb)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc composition"); }
            if ((e = dev_alloc(&c->d_mob, nb)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc mobility"); }
            if ((e = dev_alloc(&c->d_tcond, (size_t)c->stride * sizeof(double))) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc conductivity"); }
        }
    }
    {
        double *t0 = (double *)malloc((size_t)p->npf * sizeof(double));
        if (!t0) { free_ctx(c); return set_error(CIPHER_E_NOMEM, "host allocation"); }
        for (int a = 0; a < p->npf; a++) t0[a] = p->material[p->phasematerialmapping[a]].temperature0;
        e = dev_alloc(&c->d_t0, (size_t)p->npf * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpy(c->d_t0, t0, (size_t)p->npf * sizeof(double), cudaMemcpyHostToDevice);
        free(t0);
        if (e != cudaSuccess) { free_ctx(c); return cuda_fail(e, "temperature table"); }
    }
    if ((e = dev_alloc(&c->d_pruned, (size_t)(c->P + 1) * c->stride * sizeof(uint16_t))) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc pruned"); }
    if (c->aniso && (e = dev_alloc(&c->d_grad, (size_t)c->dim * c->P * c->stride * sizeof(double))) != cudaSuccess) {
        free_ctx(c);
        return cuda_fail(e, "cudaMalloc gradients");
    }
    /* the FP64 reference-order kernel groups cells by set size above a
     * 128^2 grid (on smaller domains the grouping's launches cost more than
     * the lane activity gains) */
    const bool order_pf = !c->general && c->precision == CIPHER_PREC_FP64 && c->P < kOrderClasses &&
                          c->ncells > kSpecialisedMinCells;
    if ((c->general && c->nmat + 3 <= kOrderClasses) || order_pf) {
        c->nclass = c->general ? c->nmat + 3 : c->P + 1;
        const size_t nblk = (size_t)(c->ncells + 255) / 256;
        if ((e = dev_alloc(&c->d_order, (size_t)c->stride * sizeof(int32_t))) != cudaSuccess ||
            (e = dev_alloc(&c->d_order_cursor, kOrderClasses * sizeof(int32_t))) != cudaSuccess ||
            (e = dev_alloc(&c->d_order_counts, kOrderClasses * nblk * sizeof(int32_t))) != cudaSuccess) {
            free_ctx(c);
            return cuda_fail(e, "cudaMalloc cell order");
        }
    }
    /* Specialised chemistry kernels, each giving the same bits as the
     * general kernels (CIPHER_B200_SPECIALISED_KERNELS=0 keeps every cell in
     * the general kernels, =1 uses the specialised ones at any size, to
     * compare the two):
     *  - single-phase cells, per model whose materials all have the model's
     *    sublattice count, compiled for 2..5 components (rhs_single.cu);
     *  - the phases of cells of several phases as (cell, phase) items, one
     *    thread each (rhs_items.cu), compiled for the component count and
     *    model when every material has the same model (not "none"). */
    c->item_model = -1;
    /* by default only above a 128^2 grid: on smaller domains the extra
     * launches cost more than the specialised kernels save */
    const char *spec_env = getenv("CIPHER_B200_SPECIALISED_KERNELS");
    const bool spec_on = spec_env && strcmp(spec_env, "1") == 0 ? true
                         : spec_env && strcmp(spec_env, "0") == 0 ? false
                                                                   : c->ncells > kSpecialisedMinCells;
    if (spec_on && c->general && c->d_order && c->ncp >= 2 && c->ncp <= 5) {
        uint32_t present = 0, bad = 0;
        for (int m = 0; m < p->nmat; m++) {
            const int model = p->material[m].model;
            if (model < 0 || model >= 32) { bad = ~0u; break; }
            present |= 1u << model;
            if (p->material[m].nsites != model_nsites(model)) bad |= 1u << model;
        }
        c->single_models = present & ~bad;
        if (c->single_models == present && (present & (present - 1)) == 0 && present != (1u << CIPHER_CHEM_NONE))
            c->item_model = __builtin_ctz(present);
    }
    if (spec_on && c->general && c->d_order && c->ndp > 0 && c->ncells < ((int64_t)1 << 27)) {
        /* room for the items of a few cells in ten, else those cells are
         * evaluated whole by the general kernel */
        int64_t cap = c->ncells / 2 > 65536 ? c->ncells / 2 : 65536;
        if (cap > c->ncells * c->P) cap = c->ncells * c->P;
        /* CIPHER_B200_ITEM_CAPACITY=N caps the items (less device memory;
         * the cells that do not fit are evaluated whole) */
        const char *cap_env = getenv("CIPHER_B200_ITEM_CAPACITY");
        if (cap_env && atoll(cap_env) > 0 && atoll(cap_env) < cap) cap = atoll(cap_env);
        const int nq = item_q(c->ndp, c->S).nq;
        if ((e = dev_alloc(&c->d_ibase, (size_t)c->stride * sizeof(int32_t))) != cudaSuccess ||
            (e = dev_alloc(&c->d_icell, (size_t)cap * sizeof(int32_t))) != cudaSuccess ||
            (e = dev_alloc(&c->d_icount, sizeof(int32_t))) != cudaSuccess ||
            (e = dev_alloc(&c->d_iscr, (size_t)nq * cap * sizeof(double))) != cudaSuccess) {
            free_ctx(c);
            return cuda_fail(e, "cudaMalloc phase items");
        }
        /* every entry names no item until a listing writes it */
        if ((e = cudaMemset(c->d_icell, 0xff, (size_t)cap * sizeof(int32_t))) != cudaSuccess ||
            (e = cudaStreamSynchronize(0)) != cudaSuccess) {
            free_ctx(c);
            return cuda_fail(e, "cudaMemset phase items");
        }
        c->icap = cap;
    }
    if ((e = dev_alloc(&c->d_err, sizeof(int))) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMalloc err"); }
    if ((e = cudaMemset(c->d_err, 0, sizeof(int))) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "cudaMemset err"); }
    if ((e = pinned_word_alloc(&c->h_err)) != cudaSuccess) { free_ctx(c); return cuda_fail(e, "pinned error word"); }
    if (c->listed) {
        int rc = upload_face_lists(c, m, p->dim);
        if (rc) { free_ctx(c); return rc; }
    }
    *c->h_err = 0;
    *out = c;
    return CIPHER_OK;
}

extern "C" void cipher_ctx_destroy(cipher_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    free_ctx(c);
}

extern "C" int cipher_ctx_layout(const cipher_ctx *c, cipher_state_layout *out)
{
    if (!c || !out) return set_error(CIPHER_E_ARG, "NULL argument");
    *out = c->lay;
    return CIPHER_OK;
}

/* ------------------------------------------------------------------ */
/* RHS and PostStep                                                     */
/* ------------------------------------------------------------------ */

/* largest float whose double value is <= x, smallest whose value is >= x */
static float float_at_most(double x)
{
    float f = (float)x;
    return (double)f > x ? nextafterf(f, -INFINITY) : f;
}
static float float_at_least(double x)
{
    float f = (float)x;
    return (double)f < x ? nextafterf(f, INFINITY) : f;
}

template <typename R>
static void mixed_consts(PfArgs<R> &a)
{
    const double pi2 = CIPHER_PI_D * CIPHER_PI_D;
    a.sig_f = (float)a.sig0;
    a.inv_w_f = (float)(1.0 / a.wid0);
    a.w_pi2_f = (float)(a.wid0 / pi2);
    a.tjh_f = (float)(0.5 * a.tj0);
    a.mob_f = (float)a.mob0;
    a.coef_f = (float)a.face_coef;
    a.tol_gt = float_at_most(CIPHER_TOL);
    a.tol1_lt = float_at_least(1.0 - CIPHER_TOL);
    a.tol_lt = float_at_least(CIPHER_TOL);
    a.tol1_gt = float_at_most(1.0 - CIPHER_TOL);
}

template <typename R>
static PfArgs<R> pf_args(const cipher_ctx *c, const void *X, void *F)
{
    PfArgs<R> a;
    memset(&a, 0, sizeof(a));
    const char *x = (const char *)X;
    char *f = (char *)F;
    if (!c->general) {
        a.order = c->d_order;
        a.order_cursor = c->d_order_cursor;
        a.order_counts = c->d_order_counts;
    }
    a.ncells = c->ncells;
    a.stride = c->stride;
    for (int d = 0; d < 3; d++) { a.res[d] = c->res[d]; a.per[d] = c->per[d]; }
    a.P = c->P;
    a.npf = c->npf;
    a.ffactor = c->ffactor;
    a.vol = c->vol;
    {
        int ex;
        double mant = frexp(c->vol, &ex);
        if (c->ffactor == 1.0 && c->vol == 1.0) a.geom_mode = 2;        /* GEOM_UNIT */
        else if (mant == 0.5) a.geom_mode = 1;                          /* GEOM_RECIP */
        else a.geom_mode = 0;                                           /* GEOM_DIVIDE */
        a.inv_vol = 1.0 / c->vol;
        a.face_coef = c->ffactor / c->vol;
    }
    a.junctionpenalty = c->junctionpenalty;
    a.has_temp_rate = c->has_temp_rate;
    a.temp_rate = c->temp_rate;
    a.single = c->single;
    a.sig0 = c->sig0;
    a.mob0 = c->mob0;
    a.wid0 = c->wid0;
    a.tj0 = c->tj0;
    mixed_consts(a);
    a.itflist = c->d_itflist;
    a.itfs = c->d_itfs;
    a.as = (const uint16_t *)(x + c->lay.as_offset);
    a.maps = (const uint32_t *)(x + c->lay.map_offset);
    a.phi = (const R *)(x + c->lay.pf_offset);
    a.tm = (const R *)(x + c->lay.tm_offset);
    a.fphi = (R *)(f + c->lay.pf_offset);
    a.ftm = (R *)(f + c->lay.tm_offset);
    a.err = c->d_err;
    return a;
}

template <typename R>
static GenArgs<R> gen_args(const cipher_ctx *c, const void *X, void *F)
{
    GenArgs<R> a;
    memset(&a, 0, sizeof(a));
    const char *x = (const char *)X;
    char *f = (char *)F;
    a.ncells = c->ncells;
    a.stride = c->stride;
    for (int d = 0; d < 3; d++) { a.res[d] = c->res[d]; a.per[d] = c->per[d]; }
    a.P = c->P;
    a.npf = c->npf;
    a.ncp = c->ncp;
    a.ndp = c->ndp;
    a.SP = c->S;
    a.interp = c->interp;
    a.ffactor = c->ffactor;
    a.vol = c->vol;
    {
        int ex;
        double mant = frexp(c->vol, &ex);
        if (c->ffactor == 1.0 && c->vol == 1.0) a.geom_mode = 2;
        else if (mant == 0.5) a.geom_mode = 1;
        else a.geom_mode = 0;
        a.inv_vol = 1.0 / c->vol;
    }
    a.delta = c->delta;
    a.junctionpenalty = c->junctionpenalty;
    a.has_temp_rate = c->has_temp_rate;
    a.temp_rate = c->temp_rate;
    a.itflist = c->d_itflist;
    a.itfs = c->d_itfs;
    a.chem.mat = c->d_mat;
    a.chem.pmm = c->d_pmm;
    a.chem.ncp = c->ncp;
    a.chem.ndp = c->ndp;
    a.chem.nmat = c->nmat;
    a.chem.spec = c->d_mat_spec;
    a.chem.tspec = c->d_tspec;
    a.chem.matv_tab = c->d_matv;
    a.nbcs = c->nbcs;
    for (int b = 0; b < c->nbcs; b++) a.bcs[b] = c->bcs[b];
    a.as = (const uint16_t *)(x + c->lay.as_offset);
    a.phi = (const R *)(x + c->lay.pf_offset);
    a.dp = (const double *)(x + c->lay.dp_offset);
    a.ex = (const double *)(x + c->lay.ex_offset);
    a.tm = (const R *)(x + c->lay.tm_offset);
    a.fl = face_lists(c);
    a.grad = c->d_grad;
    a.order = c->d_order;
    a.order_cursor = c->d_order_cursor;
    a.order_counts = c->d_order_counts;
    a.nclass = c->nclass;
    a.single_models = c->single_models;
    if (c->icap) {
        a.iscr = c->d_iscr;
        a.ibase = c->d_ibase;
        a.icell = c->d_icell;
        a.icount = c->d_icount;
        a.icap = c->icap;
    }
    a.item_model = c->item_model;
    for (int d = 0; d < 3; d++) a.cw[d] = c->cw[d];
    a.comp = c->d_comp;
    a.mob = c->d_mob;
    a.tcond = c->d_tcond;
    if (f) {
        a.fphi = (R *)(f + c->lay.pf_offset);
        a.fdp = (double *)(f + c->lay.dp_offset);
        a.fex = (double *)(f + c->lay.ex_offset);
        a.ftm = (R *)(f + c->lay.tm_offset);
    }
    a.err = c->d_err;
    return a;
}

extern "C" int cipher_rhs(cipher_ctx *c, double t, const void *X, void *F, void *stream)
{
    (void)t;
    if (!c || !X || !F) return set_error(CIPHER_E_ARG, "NULL argument");
    if (X == F) return set_error(CIPHER_E_ARG, "X and F must not alias");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (c->general) {
        if (c->precision == CIPHER_PREC_FP64) e = launch_rhs_general(gen_args<double>(c, X, F), c->dim, s);
        else e = launch_rhs_general(gen_args<float>(c, X, F), c->dim, s);
    } else if (c->precision == CIPHER_PREC_FP64) {
        if (c->rhs_form == CIPHER_RHS_CLOSED_FORM && c->single)
            e = launch_rhs_items_fp64(pf_args<double>(c, X, F), c->dim, s);
        else
            e = launch_rhs_phasefield(pf_args<double>(c, X, F), c->dim, s);
    } else {
        e = launch_rhs_phasefield(pf_args<float>(c, X, F), c->dim, s);
    }
    if (e != cudaSuccess) return cuda_fail(e, "rhs launch");
    return CIPHER_OK;
}

extern "C" int cipher_ctx_set_rhs_form(cipher_ctx *c, int form)
{
    if (!c) return set_error(CIPHER_E_ARG, "NULL context");
    if (form != CIPHER_RHS_REFERENCE_ORDER && form != CIPHER_RHS_CLOSED_FORM)
        return set_error(CIPHER_E_ARG, "unknown RHS form %d", form);
    c->rhs_form = form;
    return CIPHER_OK;
}

template <typename R>
static PostArgs<R> post_args(const cipher_ctx *c, void *X)
{
    PostArgs<R> a;
    memset(&a, 0, sizeof(a));
    char *x = (char *)X;
    a.ncells = c->ncells;
    a.stride = c->stride;
    for (int d = 0; d < 3; d++) { a.res[d] = c->res[d]; a.per[d] = c->per[d]; }
    a.P = c->P;
    a.S = c->S;
    a.as = (uint16_t *)(x + c->lay.as_offset);
    /* adapted meshes have no face maps (their general kernels merge sets) */
    a.maps = c->lay.map_planes ? (uint32_t *)(x + c->lay.map_offset) : nullptr;
    a.fl = face_lists(c);
    a.npf = c->npf;
    a.phi = (R *)(x + c->lay.pf_offset);
    a.ex = (double *)(x + c->lay.ex_offset);
    a.tm = (const R *)(x + c->lay.tm_offset);
    a.pruned = c->d_pruned;
    a.chem.mat = c->d_mat;
    a.chem.pmm = c->d_pmm;
    a.chem.ncp = c->ncp;
    a.chem.ndp = c->ndp;
    a.chem.nmat = c->nmat;
    a.err = c->d_err;
    return a;
}

/* ------------------------------------------------------------------ */
/* internal accessors for the batch driver (batch.cu)                   */
/* ------------------------------------------------------------------ */

namespace cipher {
CtxInfo ctx_info(const cipher_ctx *c)
{
    CtxInfo i;
    i.device = c->device;
    i.precision = c->precision;
    i.dim = c->dim;
    i.general = c->general;
    i.single = c->single;
    i.listed = c->listed;
    i.P = c->P;
    i.ncells = c->ncells;
    i.res[0] = c->res[0]; i.res[1] = c->res[1]; i.res[2] = c->res[2];
    return i;
}
PfArgs<double> ctx_pf_args_d(const cipher_ctx *c, const void *X, void *F, int *err)
{
    PfArgs<double> a = pf_args<double>(c, X, F);
    a.err = err;
    return a;
}
PfArgs<float> ctx_pf_args_f(const cipher_ctx *c, const void *X, void *F, int *err)
{
    PfArgs<float> a = pf_args<float>(c, X, F);
    a.err = err;
    return a;
}
PostArgs<double> ctx_post_args_d(const cipher_ctx *c, void *X, uint16_t *pruned, int *err)
{
    PostArgs<double> a = post_args<double>(c, X);
    a.pruned = pruned;
    a.err = err;
    return a;
}
PostArgs<float> ctx_post_args_f(const cipher_ctx *c, void *X, uint16_t *pruned, int *err)
{
    PostArgs<float> a = post_args<float>(c, X);
    a.pruned = pruned;
    a.err = err;
    return a;
}
GenArgs<double> ctx_gen_args_d(const cipher_ctx *c, const void *X) { return gen_args<double>(c, X, nullptr); }
GenArgs<float> ctx_gen_args_f(const cipher_ctx *c, const void *X) { return gen_args<float>(c, X, nullptr); }
double ctx_cell_volume(const cipher_ctx *c) { return c->vol; }

cudaError_t ctx_rhs_general(const cipher_ctx *c, const void *X, void *F, int *err, cudaStream_t s)
{
    if (c->precision == CIPHER_PREC_FP64) {
        GenArgs<double> a = gen_args<double>(c, X, F);
        a.err = err;
        return launch_rhs_general(a, c->dim, s);
    }
    GenArgs<float> a = gen_args<float>(c, X, F);
    a.err = err;
    return launch_rhs_general(a, c->dim, s);
}
}  // namespace cipher

static int read_flags(cipher_ctx *c, cudaStream_t s, int *flags)
{
    CUDA_TRY(cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, s), "read error flags");
    CUDA_TRY(cudaStreamSynchronize(s), "stream sync");
    *flags = *c->h_err;
    if (*flags) CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), s), "clear error flags");
    return CIPHER_OK;
}

extern "C" int cipher_poststep(cipher_ctx *c, void *X, void *stream)
{
    if (!c || !X) return set_error(CIPHER_E_ARG, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (c->precision == CIPHER_PREC_FP64) e = launch_poststep(post_args<double>(c, X), c->dim, s);
    else e = launch_poststep(post_args<float>(c, X), c->dim, s);
    if (e != cudaSuccess) return cuda_fail(e, "poststep launch");
    int flags = 0;
    int rc = read_flags(c, s, &flags);
    if (rc) return rc;
    if (flags & ERR_CAP) return set_error(CIPHER_E_CAP, "active-set superset exceeds the cap P=%d", c->P);
    if (flags & ERR_BADSET) return set_error(CIPHER_E_ARG, "state holds an active count outside 1..P");
    return CIPHER_OK;
}

/* explicit site potentials and chemical potentials of an initial state
 * whose sets, phi and T are filled (src/init.c:1790-1823) */
extern "C" int cipher_chem_init(cipher_ctx *c, void *X, void *stream)
{
    if (!c || !X) return set_error(CIPHER_E_ARG, "NULL argument");
    if (!c->ndp) return CIPHER_OK;
    cudaStream_t s = (cudaStream_t)stream;
    char *x = (char *)X;
    double *ex = (double *)(x + c->lay.ex_offset), *dp = (double *)(x + c->lay.dp_offset);
    cudaError_t e;
    if (c->precision == CIPHER_PREC_FP64) e = launch_chem_init(gen_args<double>(c, X, nullptr), ex, dp, s);
    else e = launch_chem_init(gen_args<float>(c, X, nullptr), ex, dp, s);
    if (e != cudaSuccess) return cuda_fail(e, "chem init launch");
    return CIPHER_OK;
}

/* sync, read and clear the kernels' error flags */
extern "C" int cipher_ctx_check(cipher_ctx *c, void *stream)
{
    if (!c) return set_error(CIPHER_E_ARG, "NULL argument");
    int flags = 0;
    int rc = read_flags(c, (cudaStream_t)stream, &flags);
    if (rc) return rc;
    if (flags & ERR_CAP) return set_error(CIPHER_E_CAP, "active-set superset exceeds the cap P=%d", c->P);
    if (flags & ERR_BADSET) return set_error(CIPHER_E_ARG, "state holds an active count outside 1..P");
    return CIPHER_OK;
}

namespace cipher {
cudaError_t launch_waxpy(int precision, int64_t nreal, int64_t ndbl, const void *xr, const void *fr, void *yr,
                         const double *xd, const double *fd, double *yd, double a, cudaStream_t s);
}

extern "C" int cipher_waxpy(cipher_ctx *c, void *Y, const void *X, double a, const void *F, void *stream)
{
    if (!c || !Y || !X || !F) return set_error(CIPHER_E_ARG, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    const char *x = (const char *)X, *f = (const char *)F;
    char *y = (char *)Y;
    const cipher_state_layout &L = c->lay;
    if (Y != X)
        CUDA_TRY(cudaMemcpyAsync(y + L.as_offset, x + L.as_offset, (size_t)(L.pf_offset - L.as_offset),
                                 cudaMemcpyDeviceToDevice, s), "copy AS");
    int64_t rb = c->precision == CIPHER_PREC_FP64 ? 8 : 4;
    int64_t nreal = (int64_t)c->P * c->stride;
    int64_t ndbl = (L.tm_offset - L.dp_offset) / 8;
    cudaError_t e = launch_waxpy(c->precision, nreal, ndbl, x + L.pf_offset, f + L.pf_offset, y + L.pf_offset,
                                 (const double *)(x + L.dp_offset), (const double *)(f + L.dp_offset),
                                 (double *)(y + L.dp_offset), a, s);
    if (e != cudaSuccess) return cuda_fail(e, "waxpy launch");
    e = launch_waxpy(c->precision, c->stride, 0, x + L.tm_offset, f + L.tm_offset, y + L.tm_offset,
                     nullptr, nullptr, nullptr, a, s);
    if (e != cudaSuccess) return cuda_fail(e, "waxpy launch");
    (void)rb;
    return CIPHER_OK;
}

/* ------------------------------------------------------------------ */
/* layouts and the host-buffer entry point                             */
/* ------------------------------------------------------------------ */

static LayoutArgs layout_args(const cipher_ctx *c, void *X)
{
    LayoutArgs a;
    memset(&a, 0, sizeof(a));
    char *x = (char *)X;
    a.ncells = c->ncells;
    a.stride = c->stride;
    a.P = c->P;
    a.D = c->ndp;
    a.E = c->P * c->S;
    a.ndof = c->aos.ndof;
    a.as_off = c->aos.as_offset;
    a.pf_off = c->aos.pf_offset;
    a.dp_off = c->aos.dp_offset;
    a.ex_off = c->aos.ex_offset;
    a.tm_off = c->aos.tm_offset;
    a.real_bytes = c->precision == CIPHER_PREC_FP64 ? 8 : 4;
    a.as = (uint16_t *)(x + c->lay.as_offset);
    a.phi = x + c->lay.pf_offset;
    a.dp = (double *)(x + c->lay.dp_offset);
    a.ex = (double *)(x + c->lay.ex_offset);
    a.tm = x + c->lay.tm_offset;
    return a;
}

static cudaError_t build_maps(const cipher_ctx *c, void *X, cudaStream_t s)
{
    if (c->precision == CIPHER_PREC_FP64) return launch_build_maps(post_args<double>(c, X), c->dim, s);
    return launch_build_maps(post_args<float>(c, X), c->dim, s);
}

extern "C" int cipher_state_from_aos(cipher_ctx *c, const double *aos, void *X, void *stream)
{
    if (!c || !aos || !X) return set_error(CIPHER_E_ARG, "NULL argument");
    cudaError_t e = launch_aos_to_soa(layout_args(c, X), aos, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "aos->state launch");
    e = build_maps(c, X, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "face map launch");
    return CIPHER_OK;
}

extern "C" int cipher_state_init_sharp(cipher_ctx *c, const int32_t *voxelphase, void *X, void *stream)
{
    if (!c || !voxelphase || !X) return set_error(CIPHER_E_ARG, "NULL argument");
    if (c->listed)
        return set_error(CIPHER_E_UNSUPPORTED, "the device initial state needs a uniform grid; build an adapted "
                                               "mesh's state on the host (cipher_initial_state_aos)");
    cudaStream_t s = (cudaStream_t)stream;
    int32_t *d_vox = nullptr;
    CUDA_TRY(dev_alloc(&d_vox, (size_t)c->ncells * sizeof(int32_t)), "voxel map");
    cudaError_t e = cudaMemcpyAsync(d_vox, voxelphase, (size_t)c->ncells * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    InitArgs a;
    memset(&a, 0, sizeof(a));
    a.L = layout_args(c, X);
    for (int d = 0; d < 3; d++) { a.res[d] = c->res[d]; a.per[d] = c->per[d]; }
    a.dim = c->dim;
    a.npf = c->npf;
    a.voxel = d_vox;
    a.t0 = c->d_t0;
    a.err = c->d_err;
    if (e == cudaSuccess) e = launch_init_sharp(a, s);
    if (e == cudaSuccess) e = build_maps(c, X, s);
    if (e != cudaSuccess) { cudaStreamSynchronize(s); dev_free(d_vox); return cuda_fail(e, "initial state"); }
    int rc = cipher_chem_init(c, X, stream);
    int flags = 0;
    if (!rc) rc = read_flags(c, s, &flags);
    /* the map's readers are done once the stream is (read_flags synchronises it) */
    cudaStreamSynchronize(s);
    dev_free(d_vox);
    if (rc) return rc;
    if (flags & ERR_CAP) return set_error(CIPHER_E_CAP, "an initial active set exceeds the cap P=%d", c->P);
    if (flags & ERR_BADSET) return set_error(CIPHER_E_ARG, "voxel map holds a phase outside 0..npf-1");
    return CIPHER_OK;
}

extern "C" int cipher_output_fields(cipher_ctx *c, const void *X, const cipher_output_field *fields, int nfields,
                                    double *out, void *stream)
{
    if (!c || !X || !fields || !out || nfields < 1) return set_error(CIPHER_E_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    int32_t *h = (int32_t *)malloc((size_t)nfields * 2 * sizeof(int32_t));
    if (!h) return set_error(CIPHER_E_NOMEM, "host allocation");
    for (int k = 0; k < nfields; k++) {
        if (fields[k].kind < CIPHER_OUT_PHASEID || fields[k].kind > CIPHER_OUT_TEMPERATURE) {
            free(h);
            return set_error(CIPHER_E_ARG, "output field %d: unknown kind %d", k, fields[k].kind);
        }
        h[k] = fields[k].kind;
        h[nfields + k] = fields[k].index;
    }
    int32_t *d = nullptr;
    cudaError_t e = cudaMalloc(&d, (size_t)nfields * 2 * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, h, (size_t)nfields * 2 * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        if (c->precision == CIPHER_PREC_FP64) e = launch_output_fields(gen_args<double>(c, X, nullptr), d, d + nfields, nfields, out, s);
        else e = launch_output_fields(gen_args<float>(c, X, nullptr), d, d + nfields, nfields, out, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d);
    free(h);
    if (e != cudaSuccess) return cuda_fail(e, "output fields");
    return cipher_ctx_check(c, stream);
}

extern "C" int cipher_state_transfer(cipher_ctx *dst, void *Xdst, const cipher_ctx *src, const void *Xsrc,
                                     const int64_t *src0, const int32_t *nsrc, void *stream)
{
    if (!dst || !Xdst || !src || !Xsrc || !src0 || !nsrc) return set_error(CIPHER_E_ARG, "NULL argument");
    if (dst->device != src->device || dst->precision != src->precision || dst->P != src->P || dst->ndp != src->ndp ||
        dst->S != src->S)
        return set_error(CIPHER_E_ARG, "the two contexts differ in device, precision or state layout");
    for (int64_t i = 0; i < dst->ncells; i++)
        if (nsrc[i] < 1 || src0[i] < 0 || src0[i] + nsrc[i] > src->ncells)
            return set_error(CIPHER_E_ARG, "transfer plan entry %lld is out of range", (long long)i);
    cudaStream_t s = (cudaStream_t)stream;
    int64_t *d_s0 = nullptr;
    int32_t *d_ns = nullptr;
    cudaError_t e = dev_alloc(&d_s0, (size_t)dst->ncells * sizeof(int64_t));
    if (e == cudaSuccess) e = dev_alloc(&d_ns, (size_t)dst->ncells * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_s0, src0, (size_t)dst->ncells * sizeof(int64_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ns, nsrc, (size_t)dst->ncells * sizeof(int32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_transfer(layout_args(dst, Xdst), layout_args(src, (void *)Xsrc), d_s0, d_ns, s);
    if (e == cudaSuccess) e = build_maps(dst, Xdst, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    dev_free(d_s0);
    dev_free(d_ns);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(e, "state transfer");
    return CIPHER_OK;
}

extern "C" int cipher_state_refresh(cipher_ctx *c, void *X, void *stream)
{
    if (!c || !X) return set_error(CIPHER_E_ARG, "NULL argument");
    cudaError_t e = build_maps(c, X, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "face map launch");
    return CIPHER_OK;
}

extern "C" int cipher_state_to_aos(cipher_ctx *c, const void *X, double *aos, void *stream)
{
    if (!c || !aos || !X) return set_error(CIPHER_E_ARG, "NULL argument");
    cudaError_t e = launch_soa_to_aos(layout_args(c, (void *)X), aos, 1, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "state->aos launch");
    return CIPHER_OK;
}

static int make_pipeline(cipher_ctx *c)
{
    if (c->pipe_ready) return CIPHER_OK;
    CUDA_TRY(cudaStreamCreateWithFlags(&c->s_up, cudaStreamNonBlocking), "stream");
    CUDA_TRY(cudaStreamCreateWithFlags(&c->s_cp, cudaStreamNonBlocking), "stream");
    CUDA_TRY(cudaStreamCreateWithFlags(&c->s_dn, cudaStreamNonBlocking), "stream");
    CUDA_TRY(cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming), "event");
    CUDA_TRY(cudaEventCreateWithFlags(&c->ev_end, cudaEventDisableTiming), "event");
    for (int i = 0; i < kAosSlabs; i++) {
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_up[i], cudaEventDisableTiming), "event");
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_done[i], cudaEventDisableTiming), "event");
    }
    c->pipe_ready = 1;
    return CIPHER_OK;
}

/* phase-field RHS of 3D grids in z-slabs: slab i is copied in and converted
 * on s_up; once its own and both neighbouring slabs are in, its face maps,
 * RHS and F conversion run on s_cp and its F rows are copied out on s_dn,
 * so that copies out of finished slabs overlap copies into later ones.
 * With periodic z the last slab is copied in second, so that the slabs can
 * run in order with each waiting for one more copy. */
template <typename R>
static int aos_host_slabs(cipher_ctx *c, const double *X_host, double *F_host, cudaStream_t s)
{
    int rc = make_pipeline(c);
    if (rc) return rc;
    const int Rz = c->res[2];
    const int K = Rz < kAosSlabs ? Rz : kAosSlabs;
    const int64_t plane = (int64_t)c->res[0] * c->res[1];
    const int64_t ndof = c->aos.ndof;
    int zs[kAosSlabs + 1];
    for (int i = 0; i <= K; i++) zs[i] = (int)((int64_t)Rz * i / K);
    const bool wrap = c->per[2] && Rz > 1;
    CUDA_TRY(cudaEventRecord(c->ev_start, s), "event");
    CUDA_TRY(cudaStreamWaitEvent(c->s_up, c->ev_start, 0), "wait");
    CUDA_TRY(cudaStreamWaitEvent(c->s_cp, c->ev_start, 0), "wait");
    CUDA_TRY(cudaStreamWaitEvent(c->s_dn, c->ev_start, 0), "wait");
    const LayoutArgs lx = layout_args(c, c->d_X), lf = layout_args(c, c->d_F);
    cudaError_t e;
    for (int u = 0; u < K; u++) {
        const int i = !wrap || u == 0 ? u : u == 1 ? K - 1 : u - 1;   /* periodic: 0, K-1, 1, 2, ... */
        const int64_t c0 = zs[i] * plane, c1 = zs[i + 1] * plane;
        CUDA_TRY(cudaMemcpyAsync(c->d_aos_x + c0 * ndof, X_host + c0 * ndof, (size_t)((c1 - c0) * ndof) * sizeof(double),
                                 cudaMemcpyHostToDevice, c->s_up), "copy X slab to device");
        if ((e = launch_aos_to_soa_range(lx, c->d_aos_x, c0, c1, c->s_up)) != cudaSuccess) return cuda_fail(e, "aos->state launch");
        CUDA_TRY(cudaEventRecord(c->ev_up[i], c->s_up), "event");
    }
    for (int i = 0; i < K; i++) {
        for (int d = -1; d <= 1; d++) {
            int j = i + d;
            if (j < 0 || j >= K) {
                if (!wrap) continue;
                j = (j + K) % K;
            }
            CUDA_TRY(cudaStreamWaitEvent(c->s_cp, c->ev_up[j], 0), "wait");
        }
        const int64_t c0 = zs[i] * plane, c1 = zs[i + 1] * plane;
        if ((e = launch_build_maps_range(post_args<R>(c, c->d_X), 3, c0, c1, c->s_cp)) != cudaSuccess)
            return cuda_fail(e, "face map launch");
        PfArgs<R> a = pf_args<R>(c, c->d_X, c->d_F);
        a.zbase = zs[i];
        a.zcount = zs[i + 1] - zs[i];
        if ((e = launch_rhs_phasefield(a, 3, c->s_cp)) != cudaSuccess) return cuda_fail(e, "rhs launch");
        if ((e = launch_soa_to_aos_range(lf, c->d_aos_f, 0, c0, c1, c->s_cp)) != cudaSuccess)
            return cuda_fail(e, "state->aos launch");
        CUDA_TRY(cudaEventRecord(c->ev_done[i], c->s_cp), "event");
        CUDA_TRY(cudaStreamWaitEvent(c->s_dn, c->ev_done[i], 0), "wait");
        CUDA_TRY(cudaMemcpyAsync(F_host + c0 * ndof, c->d_aos_f + c0 * ndof, (size_t)((c1 - c0) * ndof) * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->s_dn), "copy F slab to host");
    }
    CUDA_TRY(cudaEventRecord(c->ev_end, c->s_dn), "event");
    CUDA_TRY(cudaStreamWaitEvent(s, c->ev_end, 0), "wait");
    return CIPHER_OK;
}

extern "C" int cipher_rhs_aos_host(cipher_ctx *c, double t, const double *X_host, double *F_host, void *stream)
{
    if (!c || !X_host || !F_host) return set_error(CIPHER_E_ARG, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    size_t nb = (size_t)c->ncells * c->aos.ndof * sizeof(double);
    if (!c->d_aos_x) {
        CUDA_TRY(dev_alloc(&c->d_aos_x, nb), "cudaMalloc aos x");
        CUDA_TRY(dev_alloc(&c->d_aos_f, nb), "cudaMalloc aos f");
        CUDA_TRY(dev_alloc(&c->d_X, (size_t)c->lay.bytes), "cudaMalloc X");
        CUDA_TRY(dev_alloc(&c->d_F, (size_t)c->lay.bytes), "cudaMalloc F");
        CUDA_TRY(cudaMemsetAsync(c->d_F, 0, (size_t)c->lay.bytes, s), "cudaMemset F");
    }
    if (!c->general && c->dim == 3 && c->res[2] >= 4) {
        /* 3D phase field: z-slab pipeline */
        const int rc = c->precision == CIPHER_PREC_FP64 ? aos_host_slabs<double>(c, X_host, F_host, s)
                                                        : aos_host_slabs<float>(c, X_host, F_host, s);
        if (rc) return rc;
    } else {
        CUDA_TRY(cudaMemcpyAsync(c->d_aos_x, X_host, nb, cudaMemcpyHostToDevice, s), "copy X to device");
        cudaError_t e = launch_aos_to_soa(layout_args(c, c->d_X), c->d_aos_x, s);
        if (e != cudaSuccess) return cuda_fail(e, "aos->state launch");
        e = build_maps(c, c->d_X, s);
        if (e != cudaSuccess) return cuda_fail(e, "face map launch");
        int rc = cipher_rhs(c, t, c->d_X, c->d_F, stream);
        if (rc) return rc;
        e = launch_soa_to_aos(layout_args(c, c->d_F), c->d_aos_f, 0, s);
        if (e != cudaSuccess) return cuda_fail(e, "state->aos launch");
        CUDA_TRY(cudaMemcpyAsync(F_host, c->d_aos_f, nb, cudaMemcpyDeviceToHost, s), "copy F to host");
    }
    CUDA_TRY(cudaStreamSynchronize(s), "stream sync");
    return cipher_ctx_check(c, stream);
}
