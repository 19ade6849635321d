/*
 * nucleation.cu - host side of nucleation on the device (the first part of
 * the reference's PostStep, src/cipher.c:715-867, with the event models of
 * src/material.c:47-128).
 *
 * Per update: the device computes, for every cell of every active site, the
 * matrix check, the nucleation barrier, the temperature and the
 * diffusivities of the site's nucleus model, and sums them per site in the
 * sites' cell order (rhs_general.cu: k_nuc_cells, k_nuc_sites).  The host
 * retires sites whose cells hold a non-matrix phase, averages the sums over
 * the site volume, and draws each remaining site's event; the device then
 * turns the cells of fired sites into their phase (k_nuc_reset).  The draws
 * come from a splitmix64 stream of the object's seed, so an update is
 * reproducible (the reference calls rand()).
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "kernels.h"

using namespace cipher;

int cipher_set_error(int code, const char *fmt, ...);

/* physical constants of the event models (src/material.c:14-15) */
static const double kAngstrom = 1.0e-10, kKbAngst2 = 1.38064852E-3;
static const double kPi = 3.14159265358979323846264338327950288419716939937510582;

struct cipher_nucleation {
    cipher_ctx *ctx;
    CtxInfo info;
    int nsites, nnuclei;
    int64_t nlist;
    std::vector<int32_t> sitephase, sitenucleus;
    std::vector<cipher_nucleus> nuclei;
    std::vector<int8_t> active, fired;
    std::vector<double> siterec, barrier, diffusivity, temperature, volume;
    uint64_t rng;
    /* device */
    int32_t *d_list, *d_site_of, *d_sitephase, *d_sitenucleus;
    int64_t *d_start;
    cipher_nucleus *d_nuclei;
    int8_t *d_active, *d_fired;
    double *d_cellrec, *d_siterec;
};

static double next_uniform(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* NucleationEvent_cnt / _constant / _thermal (src/material.c:47-119) */
static int event(const cipher_nucleus &nz, int dim, double t, double dt, double T, double volume, double gv,
                 double diffusivity, uint64_t *rng)
{
    if (nz.model == CIPHER_NUC_CONSTANT) {
        const double u = next_uniform(rng);
        return u < dt * nz.nucleation_rate && t > nz.incubationtimemin;
    }
    if (nz.model != CIPHER_NUC_CNT && nz.model != CIPHER_NUC_THERMAL) return 0;
    if (t < nz.incubationtimemin || T > nz.liquidus) return 0;
    const double KbT = kKbAngst2 * T;
    const double radius_c = 2.0 * nz.gamma / gv / kAngstrom;
    if (radius_c < nz.lengthscale * pow(volume, 1.0 / dim) && radius_c > nz.minsize) {
        const double zeldovich = nz.atomicvolume * sqrt(nz.gamma / KbT) / (2.0 * kPi * radius_c * radius_c);
        const double beta = 4.0 * kPi * diffusivity * nz.lengthscale * nz.lengthscale * radius_c / nz.atomicvolume;
        const double prob = exp(-(4.0 * kPi * nz.gamma * radius_c * radius_c) * nz.shapefactor / (3.0 * KbT));
        const double site_probability = dt * zeldovich * beta * prob;
        const double u = next_uniform(rng);
        if (u < site_probability) return 1;
    }
    return 0;
}

static void free_nu(cipher_nucleation *nu)
{
    if (!nu) return;
    cudaFree(nu->d_list);
    cudaFree(nu->d_site_of);
    cudaFree(nu->d_sitephase);
    cudaFree(nu->d_sitenucleus);
    cudaFree(nu->d_start);
    cudaFree(nu->d_nuclei);
    cudaFree(nu->d_active);
    cudaFree(nu->d_fired);
    cudaFree(nu->d_cellrec);
    cudaFree(nu->d_siterec);
    delete nu;
}

extern "C" int cipher_nucleation_create(cipher_ctx *c, int nsites, const int32_t *voxelsite, const int32_t *sitephase,
                                        const int32_t *sitenucleus, int nnuclei, const cipher_nucleus *nuclei,
                                        uint64_t seed, cipher_nucleation **out)
{
    if (!c || !out || nsites < 0 || (nsites > 0 && (!voxelsite || !sitephase || !sitenucleus || !nuclei || nnuclei < 1)))
        return cipher_set_error(CIPHER_E_ARG, "bad nucleation arguments");
    *out = NULL;
    CtxInfo info = ctx_info(c);
    if (info.listed)
        return cipher_set_error(CIPHER_E_UNSUPPORTED, "nucleation sites average over uniform cells; the context's "
                                                      "mesh is adapted");
    for (int i = 0; i < nsites; i++)
        if (sitenucleus[i] < 0 || sitenucleus[i] >= nnuclei || sitephase[i] < 0)
            return cipher_set_error(CIPHER_E_ARG, "site %d: bad nucleus or phase", i);
    for (int k = 0; k < nnuclei; k++) {
        if (nuclei[k].nmatrix < 0 || nuclei[k].nmatrix > 16) return cipher_set_error(CIPHER_E_ARG, "nucleus %d: bad matrix list", k);
        for (int j = 1; j < nuclei[k].nmatrix; j++)
            if (nuclei[k].matrix[j] <= nuclei[k].matrix[j - 1]) return cipher_set_error(CIPHER_E_ARG, "nucleus %d: matrix list not sorted", k);
    }
    cipher_nucleation *nu = new (std::nothrow) cipher_nucleation();
    if (!nu) return cipher_set_error(CIPHER_E_NOMEM, "host allocation");
    nu->ctx = c;
    nu->info = info;
    nu->nsites = nsites;
    nu->nnuclei = nnuclei;
    nu->sitephase.assign(sitephase, sitephase + nsites);
    nu->sitenucleus.assign(sitenucleus, sitenucleus + nsites);
    nu->nuclei.assign(nuclei, nuclei + nnuclei);
    nu->active.assign(nsites, 1);
    nu->fired.assign(nsites, 0);
    nu->barrier.assign(nsites, NAN);
    nu->diffusivity.assign(nsites, NAN);
    nu->temperature.assign(nsites, NAN);
    nu->volume.assign(nsites, NAN);
    nu->rng = seed;
    /* cells grouped by site, in cell order within a site (counting sort) */
    std::vector<int64_t> start(nsites + 1, 0);
    for (int64_t cell = 0; cell < info.ncells; cell++) {
        const int s = voxelsite[cell];
        if (s >= 0 && s < nsites) start[s + 1]++;
    }
    for (int s = 0; s < nsites; s++) start[s + 1] += start[s];
    nu->nlist = start[nsites];
    std::vector<int32_t> list(nu->nlist > 0 ? nu->nlist : 1), site_of(nu->nlist > 0 ? nu->nlist : 1);
    {
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (int64_t cell = 0; cell < info.ncells; cell++) {
            const int s = voxelsite[cell];
            if (s < 0 || s >= nsites) continue;
            list[fill[s]] = (int32_t)cell;
            site_of[fill[s]++] = s;
        }
    }
    const int ncp = ctx_gen_args_d(c, nullptr).ncp;
    cudaError_t e = cudaSuccess;
    const size_t nl = (size_t)(nu->nlist > 0 ? nu->nlist : 1), ns = (size_t)(nsites > 0 ? nsites : 1);
#define NU_ALLOC(ptr, bytes) if (e == cudaSuccess) e = cudaMalloc(&ptr, bytes)
    NU_ALLOC(nu->d_list, nl * sizeof(int32_t));
    NU_ALLOC(nu->d_site_of, nl * sizeof(int32_t));
    NU_ALLOC(nu->d_start, (ns + 1) * sizeof(int64_t));
    NU_ALLOC(nu->d_sitephase, ns * sizeof(int32_t));
    NU_ALLOC(nu->d_sitenucleus, ns * sizeof(int32_t));
    NU_ALLOC(nu->d_nuclei, (size_t)nnuclei * sizeof(cipher_nucleus) + 8);
    NU_ALLOC(nu->d_active, ns);
    NU_ALLOC(nu->d_fired, ns);
    NU_ALLOC(nu->d_cellrec, nl * (3 + ncp) * sizeof(double));
    NU_ALLOC(nu->d_siterec, ns * (4 + ncp) * sizeof(double));
#undef NU_ALLOC
    if (e == cudaSuccess && nu->nlist > 0) e = cudaMemcpy(nu->d_list, list.data(), nu->nlist * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nu->nlist > 0) e = cudaMemcpy(nu->d_site_of, site_of.data(), nu->nlist * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(nu->d_start, start.data(), (nsites + 1) * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nsites) e = cudaMemcpy(nu->d_sitephase, sitephase, nsites * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nsites) e = cudaMemcpy(nu->d_sitenucleus, sitenucleus, nsites * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nnuclei) e = cudaMemcpy(nu->d_nuclei, nuclei, nnuclei * sizeof(cipher_nucleus), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nsites) e = cudaMemcpy(nu->d_active, nu->active.data(), nsites, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        free_nu(nu);
        return cipher_set_error(CIPHER_E_NOMEM, "nucleation tables: %s", cudaGetErrorString(e));
    }
    nu->siterec.resize(ns * (4 + ncp));
    *out = nu;
    return CIPHER_OK;
}

extern "C" void cipher_nucleation_destroy(cipher_nucleation *nu) { free_nu(nu); }

static NucArgs nuc_args(const cipher_nucleation *nu)
{
    NucArgs a;
    memset(&a, 0, sizeof(a));
    a.nsites = nu->nsites;
    a.list = nu->d_list;
    a.start = nu->d_start;
    a.site_of = nu->d_site_of;
    a.sitephase = nu->d_sitephase;
    a.sitenucleus = nu->d_sitenucleus;
    a.nuclei = nu->d_nuclei;
    a.active = nu->d_active;
    a.cellrec = nu->d_cellrec;
    a.siterec = nu->d_siterec;
    a.fired = nu->d_fired;
    a.vol = ctx_cell_volume(nu->ctx);
    return a;
}

#define NU_CUDA(call, where)                                                                  \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return cipher_set_error(CIPHER_E_CUDA, "%s: %s", where, cudaGetErrorString(e_)); \
    } while (0)

extern "C" int cipher_nucleation_step(cipher_nucleation *nu, void *X, double t, double dt, int *nfired, void *stream)
{
    if (!nu || !X) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    if (nfired) *nfired = 0;
    if (nu->nsites == 0) return CIPHER_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const bool fp64 = nu->info.precision == CIPHER_PREC_FP64;
    const NucArgs a = nuc_args(nu);
    const int ncp = ctx_gen_args_d(nu->ctx, X).ncp;
    if (fp64) NU_CUDA(launch_nucleation_sums(ctx_gen_args_d(nu->ctx, X), a, nu->nlist, s), "nucleation sums");
    else NU_CUDA(launch_nucleation_sums(ctx_gen_args_f(nu->ctx, X), a, nu->nlist, s), "nucleation sums");
    NU_CUDA(cudaMemcpyAsync(nu->siterec.data(), nu->d_siterec, nu->nsites * (4 + ncp) * sizeof(double),
                            cudaMemcpyDeviceToHost, s), "nucleation sums");
    NU_CUDA(cudaStreamSynchronize(s), "nucleation sync");
    int nf = 0, changed = 0;
    for (int site = 0; site < nu->nsites; site++) {
        nu->fired[site] = 0;
        if (!nu->active[site]) continue;
        const double *r = &nu->siterec[(size_t)site * (4 + ncp)];
        if (r[0] == 0.0) {                      /* a cell holds a phase outside the matrix */
            nu->active[site] = 0;
            changed = 1;
            continue;
        }
        const cipher_nucleus &nz = nu->nuclei[nu->sitenucleus[site]];
        double diff = CIPHER_LARGE;
        for (int c = 0; c < ncp; c++)
            if (nz.active_solutes[c]) diff = diff < r[4 + c] ? diff : r[4 + c];
        diff /= r[1];
        const double gv = r[3] / r[1], T = r[2] / r[1];
        nu->barrier[site] = gv;
        nu->diffusivity[site] = diff;
        nu->temperature[site] = T;
        nu->volume[site] = r[1];
        if (event(nz, nu->info.dim, t, dt, T, r[1], gv, diff, &nu->rng)) {
            nu->fired[site] = 1;
            nu->active[site] = 0;
            changed = 1;
            nf++;
        }
    }
    if (changed) NU_CUDA(cudaMemcpyAsync(nu->d_active, nu->active.data(), nu->nsites, cudaMemcpyHostToDevice, s), "sites");
    if (nf) {
        NU_CUDA(cudaMemcpyAsync(nu->d_fired, nu->fired.data(), nu->nsites, cudaMemcpyHostToDevice, s), "sites");
        if (fp64) NU_CUDA(launch_nucleation_reset(ctx_gen_args_d(nu->ctx, X), a, nu->nlist, s), "nucleation reset");
        else NU_CUDA(launch_nucleation_reset(ctx_gen_args_f(nu->ctx, X), a, nu->nlist, s), "nucleation reset");
        int rc = cipher_state_refresh(nu->ctx, X, stream);
        if (rc) return rc;
    }
    NU_CUDA(cudaStreamSynchronize(s), "nucleation sync");
    if (nfired) *nfired = nf;
    return cipher_ctx_check(nu->ctx, stream);
}

extern "C" int cipher_nucleation_sites(const cipher_nucleation *nu, int8_t *active, double *barrier, double *diffusivity,
                                       double *temperature, double *volume)
{
    if (!nu) return cipher_set_error(CIPHER_E_ARG, "NULL argument");
    for (int s = 0; s < nu->nsites; s++) {
        if (active) active[s] = nu->active[s];
        if (barrier) barrier[s] = nu->barrier[s];
        if (diffusivity) diffusivity[s] = nu->diffusivity[s];
        if (temperature) temperature[s] = nu->temperature[s];
        if (volume) volume[s] = nu->volume[s];
    }
    return CIPHER_OK;
}
