/*
 * oracle_nuc.c - CPU restatement of nucleation (src/cipher.c:715-867) with
 * the barrier and event models of src/material.c:47-290, for checking the
 * device version.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference draws its events with rand(); this restatement draws from
 * the same splitmix64 stream as the library (seeded by the caller), so the
 * two can be compared site by site.  Sites are reduced in cell order.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "cipher_b200.h"

#define NUC_ANGSTROM 1.0e-10
#define NUC_KBANGST2 1.38064852E-3
#define NUC_PI 3.14159265358979323846264338327950288419716939937510582

static double nuc_uniform(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* raw energy and mobility of one material (material.c Chemenergy_* and
 * CompositionMobility_* before the molar-volume scaling) */
double or_energy_raw(const cipher_material *m, const double *y, double T, int ncp);
void or_mobility_raw(const cipher_material *m, const double *y, double T, int ncp, double *M);

/* barrier and diffusivities of one cell (NucleationBarrier_*) */
static void cell_barrier(const cipher_problem *p, const cipher_nucleus *nz, int site_phase, const uint16_t *ids, int n,
                         const double *phi, const double *mu, const double *ex, double T, double *barrier,
                         double *diff)
{
    const int ncp = p->ncp, ndp = p->ndp;
    cipher_aos_layout L = or_aos_layout(p);
    const int SP = L.sp_size;
    double h[CIPHER_MAXAP], ci[CIPHER_MAXCP] = {0}, y[CIPHER_MAXAP][2 * CIPHER_MAXCP], pot[2 * CIPHER_MAXCP];
    *barrier = 0.0;
    memset(diff, 0, (size_t)ncp * sizeof(double));
    if (nz->model != CIPHER_NUC_CNT && nz->model != CIPHER_NUC_THERMAL) return;
    or_interpolant(p->interpolation, phi, n, h);
    for (int a = 0; a < n; a++)
        for (int b = a + 1; b < n; b++) {
            const cipher_interface *itf = &p->interface[p->interfacelist[ids[a] * p->npf + ids[b]]];
            if (itf->has_potential)
                for (int d = 0; d < ndp; d++) ci[d] += h[a] * h[b] * itf->potential[d];
        }
    for (int g = 0; g < n; g++) {
        const cipher_material *mat = or_material(p, ids[g]);
        for (int s = 0; s < mat->nsites; s++)
            for (int d = 0; d < ndp; d++)
                pot[s * ndp + d] = mat->stoichiometry[s] * (mu[d] - ci[d]) - ex[g * SP + s * ndp + d];
        or_sitefrac(p, ids[g], pot, T, y[g]);
    }
    double mob[CIPHER_MAXCP];
    if (nz->model == CIPHER_NUC_CNT) {
        double matrixenergy = 0.0;
        for (int g = 0; g < n; g++) {
            const cipher_material *mat = or_material(p, ids[g]);
            matrixenergy += h[g] * or_energy_raw(mat, y[g], T, ncp) / mat->molarvolume;
            or_mobility_raw(mat, y[g], T, ncp, mob);
            for (int c = 0; c < ncp; c++) diff[c] += h[g] * CIPHER_R_GAS * T * mob[c];
        }
        const cipher_material *ms = or_material(p, site_phase);
        double exn[2 * CIPHER_MAXCP], yn[2 * CIPHER_MAXCP];
        or_sitepot_explicit(p, site_phase, ms->c0, T, exn);
        for (int s = 0; s < ms->nsites; s++)
            for (int d = 0; d < ndp; d++) pot[s * ndp + d] = ms->stoichiometry[s] * (mu[d] - ci[d]) - exn[s * ndp + d];
        or_sitefrac(p, site_phase, pot, T, yn);
        *barrier = matrixenergy - or_energy_raw(ms, yn, T, ncp) / ms->molarvolume;
    } else {
        double comp[CIPHER_MAXCP];
        for (int c = 0; c < ncp; c++) {
            comp[c] = 0.0;
            for (int g = 0; g < n; g++) {
                const cipher_material *mat = or_material(p, ids[g]);
                double avg = 0.0;
                for (int s = 0; s < mat->nsites; s++) avg += mat->stoichiometry[s] * y[g][s * ncp + c];
                comp[c] += h[g] * avg;
            }
        }
        double solvus = nz->solvus_temperature_0, enthalpy = nz->enthalpy_fusion_0;
        if (nz->has_solvus_c)
            for (int c = 0; c < ncp; c++) solvus += comp[c] * nz->solvus_temperature_c[c];
        if (nz->has_enthalpy_c)
            for (int c = 0; c < ncp; c++) enthalpy += comp[c] * nz->enthalpy_fusion_c[c];
        *barrier = enthalpy * (1.0 - T / solvus);
        for (int g = 0; g < n; g++) {
            const cipher_material *mat = or_material(p, ids[g]);
            or_mobility_raw(mat, y[g], T, ncp, mob);
            for (int c = 0; c < ncp; c++) diff[c] += h[g] * CIPHER_R_GAS * T * mob[c];
        }
    }
}

/* the event rule of NucleationEvent_* (src/material.c:47-135) up to the
 * draw: *draw = 1 when the reference draws a number for this site, and the
 * event fires when that number is below the returned threshold */
double oracle_nucleation_threshold(const cipher_nucleus *nz, int dim, double t, double dt, double T, double volume,
                                   double gv, double diffusivity, int *draw)
{
    *draw = 0;
    if (nz->model == CIPHER_NUC_CONSTANT) {
        *draw = 1;
        return t > nz->incubationtimemin ? dt * nz->nucleation_rate : -1.0;
    }
    if (nz->model != CIPHER_NUC_CNT && nz->model != CIPHER_NUC_THERMAL) return -1.0;
    if (t < nz->incubationtimemin || T > nz->liquidus) return -1.0;
    const double KbT = NUC_KBANGST2 * T;
    const double radius_c = 2.0 * nz->gamma / gv / NUC_ANGSTROM;
    if (radius_c < nz->lengthscale * pow(volume, 1.0 / dim) && radius_c > nz->minsize) {
        const double zeldovich = nz->atomicvolume * sqrt(nz->gamma / KbT) / (2.0 * NUC_PI * radius_c * radius_c);
        const double beta = 4.0 * NUC_PI * diffusivity * nz->lengthscale * nz->lengthscale * radius_c / nz->atomicvolume;
        const double prob = exp(-(4.0 * NUC_PI * nz->gamma * radius_c * radius_c) * nz->shapefactor / (3.0 * KbT));
        *draw = 1;
        return dt * zeldovich * beta * prob;
    }
    return -1.0;
}

static int nuc_event(const cipher_nucleus *nz, int dim, double t, double dt, double T, double volume, double gv,
                     double diffusivity, uint64_t *rng)
{
    int draw;
    const double thr = oracle_nucleation_threshold(nz, dim, t, dt, T, volume, gv, diffusivity, &draw);
    if (!draw) return 0;
    return nuc_uniform(rng) < thr;
}

/* one update of the whole-domain AoS state X; active[nsites] is updated,
 * out[nsites*4] receives (barrier, diffusivity, T, volume) of evaluated
 * sites; returns the number of fired sites, or -1 */
int oracle_nucleation_step(const cipher_problem *p, const cipher_mesh *m, double *X, int nsites,
                           const int32_t *voxelsite, const int32_t *sitephase, const int32_t *sitenucleus,
                           const cipher_nucleus *nuclei, double t, double dt, uint64_t *rng, int8_t *active,
                           double *out)
{
    cipher_aos_layout L = or_aos_layout(p);
    const int ndof = L.ndof, ncp = p->ncp, SP = L.sp_size;
    const double vol = or_ipow(m->cellgeom[0], (unsigned)p->dim);
    double *sums = (double *)calloc((size_t)nsites * (4 + ncp), sizeof(double));
    int8_t *ok = (int8_t *)malloc((size_t)(nsites > 0 ? nsites : 1));
    if (!sums || !ok) { free(sums); free(ok); return -1; }
    for (int s = 0; s < nsites; s++) ok[s] = active[s];
    uint16_t ids[CIPHER_MAXAP];
    for (int c = 0; c < m->ncells; c++) {
        const int s = voxelsite[m->cell_global[c]];
        if (s < 0 || s >= nsites || !ok[s]) continue;
        const double *cell = &X[(size_t)c * ndof];
        const int n = (int)round(cell[L.as_offset]);
        for (int k = 0; k < n; k++) ids[k] = (uint16_t)round(cell[L.as_offset + 1 + k]);
        const cipher_nucleus *nz = &nuclei[sitenucleus[s]];
        int common = 0;
        for (int i = 0, j = 0; i < n && j < nz->nmatrix;) {
            if (ids[i] == nz->matrix[j]) { common++; i++; j++; }
            else if (ids[i] < nz->matrix[j]) i++;
            else j++;
        }
        if (common != n) { ok[s] = 0; continue; }
        double barrier, diff[CIPHER_MAXCP];
        const double T = cell[L.tm_offset];
        cell_barrier(p, nz, sitephase[s], ids, n, &cell[L.pf_offset], &cell[L.dp_offset], &cell[L.ex_offset], T,
                     &barrier, diff);
        double *r = &sums[(size_t)s * (4 + ncp)];
        r[1] += vol;
        r[2] += vol * T;
        r[3] += vol * barrier;
        for (int k = 0; k < ncp; k++) r[4 + k] += vol * diff[k];
    }
    int nf = 0;
    int8_t *fired = (int8_t *)calloc((size_t)(nsites > 0 ? nsites : 1), 1);
    for (int s = 0; s < nsites; s++) {
        if (!active[s]) continue;
        if (!ok[s]) { active[s] = 0; continue; }
        const double *r = &sums[(size_t)s * (4 + ncp)];
        const cipher_nucleus *nz = &nuclei[sitenucleus[s]];
        double diff = CIPHER_LARGE;
        for (int k = 0; k < ncp; k++)
            if (nz->active_solutes[k]) diff = diff < r[4 + k] ? diff : r[4 + k];
        diff /= r[1];
        const double gv = r[3] / r[1], T = r[2] / r[1];
        out[4 * s + 0] = gv;
        out[4 * s + 1] = diff;
        out[4 * s + 2] = T;
        out[4 * s + 3] = r[1];
        if (nuc_event(nz, p->dim, t, dt, T, r[1], gv, diff, rng)) { fired[s] = 1; active[s] = 0; nf++; }
    }
    for (int c = 0; c < m->ncells && nf; c++) {
        const int s = voxelsite[m->cell_global[c]];
        if (s < 0 || s >= nsites || !fired[s]) continue;
        double *cell = &X[(size_t)c * ndof];
        cell[L.as_offset] = 1.0;
        cell[L.as_offset + 1] = (double)sitephase[s];
        cell[L.pf_offset] = 1.0;
        if (p->ndp) {
            const cipher_material *ms = or_material(p, sitephase[s]);
            or_sitepot_explicit(p, sitephase[s], ms->c0, cell[L.tm_offset], &cell[L.ex_offset]);
        }
        (void)SP;
    }
    free(sums); free(ok); free(fired);
    return nf;
}
