/*
 * problem.c - host-side problem construction: parameter tables, uniform
 * finite-volume leaf meshes (full domain or a slab with a one-cell halo),
 * seeded Voronoi grain maps and the initial state.
 *
 * The initial state follows the reference's SetUpProblem (src/init.c:1721-1830):
 * each cell's active set is its voxel phase united with the voxel phases of
 * its face neighbours, phi = 1 for the own phase and 0 otherwise, and the
 * temperature is the own material's temperature0.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdio.h>
#include "cipher_problem.h"
#include "cipher_b200.h"

/* ------------------------------------------------------------------ */
/* problem allocation                                                  */
/* ------------------------------------------------------------------ */

cipher_problem *cipher_problem_new(int dim, int npf, int ncp, int nmat, int nf)
{
    if (dim < 1 || dim > 3 || npf < 1 || ncp < 1 || ncp > CIPHER_MAXCP || nmat < 1 || nf < 1)
        return NULL;
    cipher_problem *p = (cipher_problem *)calloc(1, sizeof(cipher_problem));
    if (!p) return NULL;
    p->dim = dim;
    p->npf = npf;
    p->ncp = ncp;
    p->ndp = ncp - 1;
    p->nmat = nmat;
    p->nf = nf;
    p->pf_size = npf < CIPHER_MAXAP ? npf : CIPHER_MAXAP;
    p->interpolation = CIPHER_INTERP_CUBIC;
    p->junctionpenalty = 1.0;
    p->nloadcases = 1;
    p->time[0] = 1.0;
    p->timestep0 = 1.0e-18;
    p->mintimestep = 1.0e-18;
    p->maxtimestep = 1.0;
    p->reltol = 1.0e-6;
    p->abstol = 1.0e-6;
    for (int d = 0; d < 3; d++) { p->resolution[d] = 1; p->size[d] = 1.0; }
    p->material = (cipher_material *)calloc((size_t)nmat, sizeof(cipher_material));
    p->interface = (cipher_interface *)calloc((size_t)nf, sizeof(cipher_interface));
    p->interfacelist = (int32_t *)calloc((size_t)npf * (size_t)npf, sizeof(int32_t));
    p->phasematerialmapping = (int32_t *)calloc((size_t)npf, sizeof(int32_t));
    if (!p->material || !p->interface || !p->interfacelist || !p->phasematerialmapping) {
        cipher_problem_free(p);
        return NULL;
    }
    for (int m = 0; m < nmat; m++) {
        p->material[m].model = CIPHER_CHEM_NONE;
        p->material[m].molarvolume = 1.0;
    }
    for (int i = 0; i < nf; i++) {
        p->interface[i].width = 1.0;
        p->interface[i].energy_m0 = 1.0;
        p->interface[i].mobility_m0 = 1.0;
    }
    return p;
}

void cipher_problem_free(cipher_problem *p)
{
    if (!p) return;
    free(p->material);
    free(p->interface);
    free(p->interfacelist);
    free(p->phasematerialmapping);
    free(p->voxelphase);
    free(p->centres);
    free(p);
}

int cipher_problem_finalize(cipher_problem *p)
{
    int ms = 0;
    for (int m = 0; m < p->nmat; m++) {
        cipher_material *mat = &p->material[m];
        if (mat->model == CIPHER_CHEM_NONE) mat->nsites = 0;
        else if (mat->model == CIPHER_CHEM_CALPHAD2SL) {
            mat->nsites = 2;
            mat->stoichiometry[0] = mat->p;
            mat->stoichiometry[1] = mat->q;
        } else {
            mat->nsites = 1;
            mat->stoichiometry[0] = 1.0;
        }
        if (mat->nsites > ms) ms = mat->nsites;
    }
    p->maxsites = ms;
    p->ndp = p->ncp - 1;
    if (p->pf_size < 1 || p->pf_size > CIPHER_MAXAP) return CIPHER_E_ARG;
    return 0;
}

int cipher_problem_set_cap(cipher_problem *p, int max_phase_neighbours)
{
    if (max_phase_neighbours < 1 || max_phase_neighbours > CIPHER_MAXAP) return CIPHER_E_ARG;
    p->pf_size = max_phase_neighbours < p->npf ? max_phase_neighbours : p->npf;
    return 0;
}

cipher_aos_layout cipher_problem_aos_layout(const cipher_problem *p)
{
    cipher_aos_layout L;
    int P = p->pf_size;
    L.sf_size = p->maxsites * p->ncp;
    L.sp_size = p->maxsites * p->ndp;
    L.as_offset = 0;
    L.as_size = P + 1;
    L.pf_offset = L.as_offset + L.as_size;
    L.pf_size = P;
    L.dp_offset = L.pf_offset + L.pf_size;
    L.dp_size = p->ndp;
    L.ex_offset = L.dp_offset + L.dp_size;
    L.ex_size = P * L.sp_size;
    L.tm_offset = L.ex_offset + L.ex_size;
    L.ndof = L.tm_offset + 1;
    return L;
}

/* ------------------------------------------------------------------ */
/* seeded random numbers (splitmix64)                                   */
/* ------------------------------------------------------------------ */

static uint64_t splitmix64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double cipher_rand_uniform(uint64_t *state)
{
    return (double)(splitmix64(state) >> 11) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------ */
/* Voronoi grain map on a periodic box                                  */
/* ------------------------------------------------------------------ */

/* nearest-centre assignment with a bucket grid; ties go to the lower index */
int cipher_voronoi(int dim, const int32_t *res, int ngrains, uint64_t seed, int32_t *voxel, double *centres)
{
    if (dim < 1 || dim > 3 || ngrains < 1) return CIPHER_E_ARG;
    int r[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) r[d] = res[d];
    double *cen = (double *)malloc((size_t)ngrains * 3 * sizeof(double));
    if (!cen) return CIPHER_E_NOMEM;
    uint64_t s = seed;
    for (int g = 0; g < ngrains; g++)
        for (int d = 0; d < 3; d++)
            cen[3 * g + d] = d < dim ? cipher_rand_uniform(&s) * r[d] : 0.0;
    if (centres) memcpy(centres, cen, (size_t)ngrains * 3 * sizeof(double));

    /* bucket grid with about one centre per bucket */
    int nb[3] = {1, 1, 1};
    double per = pow((double)ngrains, 1.0 / dim);
    for (int d = 0; d < dim; d++) {
        nb[d] = (int)floor(per);
        if (nb[d] < 1) nb[d] = 1;
        if (nb[d] > r[d]) nb[d] = r[d];
    }
    int nbt = nb[0] * nb[1] * nb[2];
    int *bstart = (int *)calloc((size_t)nbt + 1, sizeof(int));
    int *bitem = (int *)malloc((size_t)ngrains * sizeof(int));
    int *bof = (int *)malloc((size_t)ngrains * sizeof(int));
    if (!bstart || !bitem || !bof) { free(cen); free(bstart); free(bitem); free(bof); return CIPHER_E_NOMEM; }
    for (int g = 0; g < ngrains; g++) {
        int bi[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) {
            bi[d] = (int)(cen[3 * g + d] / r[d] * nb[d]);
            if (bi[d] >= nb[d]) bi[d] = nb[d] - 1;
        }
        bof[g] = bi[0] + nb[0] * (bi[1] + nb[1] * bi[2]);
        bstart[bof[g] + 1]++;
    }
    for (int b = 0; b < nbt; b++) bstart[b + 1] += bstart[b];
    {
        int *fill = (int *)calloc((size_t)nbt, sizeof(int));
        if (!fill) { free(cen); free(bstart); free(bitem); free(bof); return CIPHER_E_NOMEM; }
        for (int g = 0; g < ngrains; g++) bitem[bstart[bof[g]] + fill[bof[g]]++] = g;
        free(fill);
    }
    double bw[3];
    for (int d = 0; d < 3; d++) bw[d] = (double)r[d] / nb[d];
    double bwmin = 1e300;
    for (int d = 0; d < dim; d++) if (bw[d] < bwmin) bwmin = bw[d];

    long total = (long)r[0] * r[1] * r[2];
    for (long c = 0; c < total; c++) {
        int x[3] = {(int)(c % r[0]), (int)((c / r[0]) % r[1]), (int)(c / ((long)r[0] * r[1]))};
        double pt[3] = {x[0] + 0.5, x[1] + 0.5, x[2] + 0.5};
        int pb[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) {
            pb[d] = (int)(pt[d] / r[d] * nb[d]);
            if (pb[d] >= nb[d]) pb[d] = nb[d] - 1;
        }
        double best = 1e300;
        int bestg = -1;
        int maxshell = 0;
        for (int d = 0; d < dim; d++) if (nb[d] > maxshell) maxshell = nb[d];
        for (int shell = 0; shell <= maxshell; shell++) {
            /* everything beyond this shell is at least (shell)*bwmin away */
            double lim = (shell - 1) * bwmin;
            if (shell > 0 && lim > 0 && lim * lim > best) break;
            int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
            for (int d = 0; d < dim; d++) { lo[d] = -shell; hi[d] = shell; }
            for (int k = lo[2]; k <= hi[2]; k++)
            for (int j = lo[1]; j <= hi[1]; j++)
            for (int i = lo[0]; i <= hi[0]; i++) {
                int o[3] = {i, j, k};
                int onshell = 0;
                for (int d = 0; d < dim; d++) if (o[d] == -shell || o[d] == shell) onshell = 1;
                if (shell > 0 && !onshell) continue;
                int bi[3];
                for (int d = 0; d < 3; d++) {
                    int v = pb[d] + (d < dim ? o[d] : 0);
                    v %= (d < dim ? nb[d] : 1);
                    if (v < 0) v += nb[d];
                    bi[d] = v;
                }
                int b = bi[0] + nb[0] * (bi[1] + nb[1] * bi[2]);
                for (int t = bstart[b]; t < bstart[b + 1]; t++) {
                    int g = bitem[t];
                    double dd = 0.0;
                    for (int d = 0; d < dim; d++) {
                        double dx = fabs(pt[d] - cen[3 * g + d]);
                        if (dx > r[d] - dx) dx = r[d] - dx;
                        dd += dx * dx;
                    }
                    if (dd < best || (dd == best && g < bestg)) { best = dd; bestg = g; }
                }
            }
            /* once the shell wraps the whole grid every bucket has been seen */
            int covered = 1;
            for (int d = 0; d < dim; d++) if (2 * shell + 1 < nb[d]) covered = 0;
            if (covered) break;
        }
        voxel[c] = bestg;
    }
    free(cen); free(bstart); free(bitem); free(bof);
    return 0;
}

/* ------------------------------------------------------------------ */
/* synthetic grain growth problem                                      */
/* ------------------------------------------------------------------ */

int cipher_problem_grain_growth(int dim, const int32_t *res, int ngrains, int cap, uint64_t seed,
                                double energy, double mobility, double width,
                                double molarvolume, double temperature0,
                                cipher_problem **out)
{
    *out = NULL;
    cipher_problem *p = cipher_problem_new(dim, ngrains, 1, 1, 1);
    if (!p) return CIPHER_E_NOMEM;
    for (int d = 0; d < dim; d++) {
        p->resolution[d] = res[d];
        p->size[d] = (double)res[d];
        p->periodic[d] = 1;
    }
    int rc = cipher_problem_set_cap(p, cap);
    if (rc) { cipher_problem_free(p); return rc; }
    cipher_material *m = &p->material[0];
    m->model = CIPHER_CHEM_NONE;
    m->molarvolume = molarvolume;
    m->temperature0 = temperature0;
    cipher_interface *itf = &p->interface[0];
    itf->width = width;
    itf->energy_m0 = energy;
    itf->mobility_m0 = mobility;
    /* every pair of grains meets through interface 0; every grain is material 0 */
    memset(p->interfacelist, 0, (size_t)ngrains * ngrains * sizeof(int32_t));
    memset(p->phasematerialmapping, 0, (size_t)ngrains * sizeof(int32_t));
    p->reltol = p->abstol = 1.0e-4;
    p->time[0] = 100.0;
    p->maxtimestep = 100.0;
    long total = 1;
    for (int d = 0; d < dim; d++) total *= res[d];
    p->voxelphase = (int32_t *)malloc((size_t)total * sizeof(int32_t));
    if (!p->voxelphase) { cipher_problem_free(p); return CIPHER_E_NOMEM; }
    p->centres = (double *)malloc((size_t)ngrains * 3 * sizeof(double));
    if (!p->centres) { cipher_problem_free(p); return CIPHER_E_NOMEM; }
    rc = cipher_voronoi(dim, res, ngrains, seed, p->voxelphase, p->centres);
    if (rc) { cipher_problem_free(p); return rc; }
    rc = cipher_problem_finalize(p);
    if (rc) { cipher_problem_free(p); return rc; }
    *out = p;
    return 0;
}

int cipher_problem_grain_growth_multi(int dim, const int32_t *res, int ngrains, int cap, uint64_t seed,
                                      int ninterfaces, unsigned features, cipher_problem **out)
{
    *out = NULL;
    if (ninterfaces < 1 || ninterfaces > 4096) return CIPHER_E_ARG;
    cipher_problem *base = NULL;
    int rc = cipher_problem_grain_growth(dim, res, ngrains, cap, seed, 1.0, 1.0, 4.0, 1.0e-5, 500.0, &base);
    if (rc) return rc;
    /* the same grid, voxel map and material with an interface table of its own */
    cipher_interface *itf = (cipher_interface *)calloc((size_t)ninterfaces, sizeof(cipher_interface));
    if (!itf) { cipher_problem_free(base); return CIPHER_E_NOMEM; }
    free(base->interface);
    base->interface = itf;
    base->nf = ninterfaces;
    uint64_t st = seed ^ 0x5bd1e995c0ffee11ull;
    for (int i = 0; i < ninterfaces; i++) {
        itf[i].width = (features & CIPHER_GG_WIDTHS) ? 3.0 + 2.0 * cipher_rand_uniform(&st) : 4.0;
        itf[i].energy_m0 = 0.5 + cipher_rand_uniform(&st);
        itf[i].mobility_m0 = 0.5 + cipher_rand_uniform(&st);
        if ((features & CIPHER_GG_ACTIVATION) && (i % 2 == 1)) {
            /* exp(Q/(R T)) factors (src/cipher.c:462-466) with Q in [-3000, 3000] J/mol */
            itf[i].energy_activation.n = 1;
            itf[i].energy_activation.exp[0] = 0;
            itf[i].energy_activation.coeff[0] = -3000.0 + 6000.0 * cipher_rand_uniform(&st);
            itf[i].mobility_activation.n = 1;
            itf[i].mobility_activation.exp[0] = 0;
            itf[i].mobility_activation.coeff[0] = -3000.0 + 6000.0 * cipher_rand_uniform(&st);
        }
    }
    /* the upper triangle, as the reference's parser fills it (src/init.c:1501) */
    const int npf = base->npf;
    for (int a = 0; a < npf; a++)
        for (int b = a + 1; b < npf; b++) {
            int i = (int)(cipher_rand_uniform(&st) * ninterfaces);
            base->interfacelist[a * npf + b] = i < ninterfaces ? i : ninterfaces - 1;
        }
    *out = base;
    return 0;
}

/* ------------------------------------------------------------------ */
/* uniform meshes                                                      */
/* ------------------------------------------------------------------ */

/*
 * The whole-domain grid description a device context needs, without face
 * lists: nfaces = nbfaces = 0, one cellgeom and cell_global entry.  Enough
 * for cipher_ctx_create (the device derives faces from the grid); the host
 * builders and the oracle need cipher_mesh_uniform instead.
 */
int cipher_mesh_grid(const cipher_problem *p, cipher_mesh **out)
{
    *out = NULL;
    int dim = p->dim;
    cipher_mesh *m = (cipher_mesh *)calloc(1, sizeof(cipher_mesh));
    if (!m) return CIPHER_E_NOMEM;
    m->dim = dim;
    m->uniform = 1;
    long cells = 1;
    double vol = 1.0;
    for (int d = 0; d < 3; d++) {
        int r = d < dim ? p->resolution[d] : 1;
        m->res[d] = r;
        m->periodic[d] = d < dim ? (p->periodic[d] && r > 1) : 0;
        cells *= r;
        if (d < dim) vol *= p->size[d] / r;
    }
    if (cells > 2147483647L) { free(m); return CIPHER_E_ARG; }
    m->ncells = m->nowned = (int32_t)cells;
    m->slab_lo = 0;
    m->slab_hi = m->res[dim - 1];
    m->cellgeom = (double *)malloc(sizeof(double));
    m->cell_global = (int32_t *)malloc(sizeof(int32_t));
    if (!m->cellgeom || !m->cell_global) { cipher_mesh_free(m); return CIPHER_E_NOMEM; }
    m->cellgeom[0] = pow(vol, 1.0 / dim);
    m->cell_global[0] = 0;
    *out = m;
    return 0;
}

void cipher_mesh_free(cipher_mesh *m)
{
    if (!m) return;
    free(m->face_cells);
    free(m->bface_cell);
    free(m->bface_label);
    free(m->cellgeom);
    free(m->cell_global);
    free(m);
}

/*
 * Uniform grid mesh.  slab_lo/slab_hi select owned planes along the slowest
 * axis; pass 0 and res[dim-1] for the whole domain.  Local cells are the owned
 * planes (x fastest), then the halo plane below, then the halo plane above.
 * Interior faces are enumerated as (c, c+e_d) for local cells c in local order
 * and d = 0..dim-1, keeping only faces whose two cells are both local.
 */
int cipher_mesh_uniform(const cipher_problem *p, int slab_lo, int slab_hi, cipher_mesh **out)
{
    *out = NULL;
    int dim = p->dim;
    int r[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) r[d] = p->resolution[d];
    int ax = dim - 1;
    if (slab_lo < 0 || slab_hi > r[ax] || slab_lo >= slab_hi) return CIPHER_E_ARG;
    int full = (slab_lo == 0 && slab_hi == r[ax]);
    long plane = 1;
    for (int d = 0; d < ax; d++) plane *= r[d];
    cipher_mesh *m = (cipher_mesh *)calloc(1, sizeof(cipher_mesh));
    if (!m) return CIPHER_E_NOMEM;
    m->dim = dim;
    m->uniform = 1;
    /* a periodic direction one cell wide would make a cell its own neighbour */
    for (int d = 0; d < 3; d++) { m->res[d] = r[d]; m->periodic[d] = d < dim ? (p->periodic[d] && r[d] > 1) : 0; }
    m->slab_lo = slab_lo;
    m->slab_hi = slab_hi;

    /* local planes: owned, then halo below, then halo above */
    int planes[4096 + 2];
    int nplanes = 0;
    if (slab_hi - slab_lo > 4096) { free(m); return CIPHER_E_ARG; }
    for (int z = slab_lo; z < slab_hi; z++) planes[nplanes++] = z;
    int nown_planes = nplanes;
    if (!full) {
        int below = slab_lo - 1, above = slab_hi;
        if (below < 0 && m->periodic[ax]) below += r[ax];
        if (above >= r[ax] && m->periodic[ax]) above -= r[ax];
        if (below >= 0 && below < r[ax]) planes[nplanes++] = below;
        if (above >= 0 && above < r[ax] && above != below) planes[nplanes++] = above;
    }
    m->nowned = (int32_t)(nown_planes * plane);
    m->ncells = (int32_t)(nplanes * plane);
    m->cellgeom = (double *)malloc((size_t)m->ncells * sizeof(double));
    m->cell_global = (int32_t *)malloc((size_t)m->ncells * sizeof(int32_t));
    if (!m->cellgeom || !m->cell_global) { cipher_mesh_free(m); return CIPHER_E_NOMEM; }
    /* map global plane -> local plane index (-1 if not local) */
    int *plocal = (int *)malloc((size_t)r[ax] * sizeof(int));
    if (!plocal) { cipher_mesh_free(m); return CIPHER_E_NOMEM; }
    for (int z = 0; z < r[ax]; z++) plocal[z] = -1;
    for (int i = 0; i < nplanes; i++) plocal[planes[i]] = i;

    double vol = 1.0;
    for (int d = 0; d < dim; d++) vol *= p->size[d] / r[d];
    double delta = pow(vol, 1.0 / dim);
    for (int i = 0; i < nplanes; i++)
        for (long k = 0; k < plane; k++) {
            long lc = i * plane + k;
            m->cell_global[lc] = (int32_t)(planes[i] * plane + k);
            m->cellgeom[lc] = delta;
        }

    /* interior faces */
    long maxf = (long)m->ncells * dim;
    m->face_cells = (int32_t *)malloc((size_t)maxf * 2 * sizeof(int32_t));
    long maxb = 2L * m->ncells;
    m->bface_cell = (int32_t *)malloc((size_t)maxb * sizeof(int32_t));
    m->bface_label = (int32_t *)malloc((size_t)maxb * sizeof(int32_t));
    if (!m->face_cells || !m->bface_cell || !m->bface_label) { free(plocal); cipher_mesh_free(m); return CIPHER_E_NOMEM; }
    long nf = 0, nbf = 0;
    for (long lc = 0; lc < m->ncells; lc++) {
        long g = m->cell_global[lc];
        int x[3] = {(int)(g % r[0]), (int)((g / r[0]) % r[1]), (int)(g / ((long)r[0] * r[1]))};
        for (int d = 0; d < dim; d++) {
            int y[3] = {x[0], x[1], x[2]};
            y[d] += 1;
            if (y[d] >= r[d]) {
                if (!m->periodic[d]) continue;
                y[d] -= r[d];
            }
            int zp = y[ax];
            int lp = plocal[zp];
            if (lp < 0) continue;
            long inplane = 0, mul = 1;
            for (int e = 0; e < ax; e++) { inplane += y[e] * mul; mul *= r[e]; }
            long nb = lp * plane + inplane;
            m->face_cells[2 * nf] = (int32_t)lc;
            m->face_cells[2 * nf + 1] = (int32_t)nb;
            nf++;
        }
    }
    /* boundary faces of owned cells on non-periodic sides, labelled as the
     * reference labels them from the face centroid: 2d+1 at 0, 2d+2 at size */
    for (long lc = 0; lc < m->nowned; lc++) {
        long g = m->cell_global[lc];
        int x[3] = {(int)(g % r[0]), (int)((g / r[0]) % r[1]), (int)(g / ((long)r[0] * r[1]))};
        for (int d = 0; d < dim; d++) {
            if (m->periodic[d]) continue;
            if (x[d] == 0) { m->bface_cell[nbf] = (int32_t)lc; m->bface_label[nbf] = 2 * d + 1; nbf++; }
            if (x[d] == r[d] - 1) { m->bface_cell[nbf] = (int32_t)lc; m->bface_label[nbf] = 2 * d + 2; nbf++; }
        }
    }
    free(plocal);
    m->nfaces = (int32_t)nf;
    m->nbfaces = (int32_t)nbf;
    *out = m;
    return 0;
}

/* ------------------------------------------------------------------ */
/* sorted-set union used by the initial active sets                    */
/* ------------------------------------------------------------------ */

/* out = a U b (sorted, duplicates merged); returns the size or -1 above cap */
static int set_union(uint16_t *out, const uint16_t *a, int na, const uint16_t *b, int nb, int cap)
{
    int i = 0, j = 0, n = 0;
    while (i < na || j < nb) {
        uint16_t v;
        if (j >= nb || (i < na && a[i] < b[j])) v = a[i++];
        else if (i >= na || b[j] < a[i]) v = b[j++];
        else { v = a[i]; i++; j++; }
        if (n >= cap) return -1;
        out[n++] = v;
    }
    return n;
}

/*
 * Initial state in the reference AoS layout for the cells of mesh m (owned
 * and ghost).  Models with chemistry need their explicit site potentials for
 * EX and the chemical potentials; those are filled by the device initialiser
 * (cipher_ctx_initial_state) and left zero here.
 */
int cipher_initial_state_aos(const cipher_problem *p, const cipher_mesh *m, double *X)
{
    cipher_aos_layout L = cipher_problem_aos_layout(p);
    int P = p->pf_size;
    int dim = p->dim;
    int r[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) r[d] = p->resolution[d];
    if (!p->voxelphase) return CIPHER_E_ARG;
    memset(X, 0, (size_t)m->ncells * L.ndof * sizeof(double));
    uint16_t set[CIPHER_MAXAP + 1], tmp[CIPHER_MAXAP + 1], one[1];
    for (long lc = 0; lc < m->ncells; lc++) {
        long g = m->cell_global[lc];
        int x[3] = {(int)(g % r[0]), (int)((g / r[0]) % r[1]), (int)(g / ((long)r[0] * r[1]))};
        int own = p->voxelphase[g];
        int n = 1;
        set[0] = (uint16_t)own;
        for (int d = 0; d < dim; d++) {
            for (int s = -1; s <= 1; s += 2) {
                int y[3] = {x[0], x[1], x[2]};
                y[d] += s;
                if (y[d] < 0 || y[d] >= r[d]) {
                    if (!p->periodic[d]) continue;
                    y[d] = (y[d] + r[d]) % r[d];
                }
                long ng = y[0] + (long)r[0] * (y[1] + (long)r[1] * y[2]);
                one[0] = (uint16_t)p->voxelphase[ng];
                int nn = set_union(tmp, set, n, one, 1, P);
                if (nn < 0) return CIPHER_E_CAP;
                memcpy(set, tmp, (size_t)nn * sizeof(uint16_t));
                n = nn;
            }
        }
        double *cell = &X[lc * L.ndof];
        cell[L.as_offset] = (double)n;
        for (int k = 0; k < n; k++) {
            cell[L.as_offset + 1 + k] = (double)set[k];
            cell[L.pf_offset + k] = set[k] == own ? 1.0 : 0.0;
        }
        cell[L.tm_offset] = p->material[p->phasematerialmapping[own]].temperature0;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* diffuse Voronoi state                                               */
/* ------------------------------------------------------------------ */

#define CIPHER_DIFFUSE_MAXCAND 64

/* minimum-image displacement c - x on a periodic box */
static void min_image(const double *x, const double *c, const int *r, const int32_t *per, int dim, double *v)
{
    for (int d = 0; d < dim; d++) {
        double dx = c[d] - x[d];
        if (per[d]) {
            if (dx > 0.5 * r[d]) dx -= r[d];
            else if (dx < -0.5 * r[d]) dx += r[d];
        }
        v[d] = dx;
    }
}

/* centres binned on a coarse grid for radius queries */
typedef struct {
    int nb[3];
    double bw[3];
    int *start, *item;
} bucket_grid;

static int bucket_build(bucket_grid *B, const double *cen, int n, const int *r, int dim, double target_width)
{
    memset(B, 0, sizeof(*B));
    for (int d = 0; d < 3; d++) B->nb[d] = 1;
    for (int d = 0; d < dim; d++) {
        int k = (int)floor(r[d] / target_width);
        B->nb[d] = k < 1 ? 1 : k;
    }
    for (int d = 0; d < 3; d++) B->bw[d] = (double)r[d] / B->nb[d];
    int nbt = B->nb[0] * B->nb[1] * B->nb[2];
    B->start = (int *)calloc((size_t)nbt + 1, sizeof(int));
    B->item = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    int *bof = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    int *fill = (int *)calloc((size_t)nbt, sizeof(int));
    if (!B->start || !B->item || !bof || !fill) { free(bof); free(fill); return CIPHER_E_NOMEM; }
    for (int g = 0; g < n; g++) {
        int bi[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) {
            bi[d] = (int)(cen[3 * g + d] / B->bw[d]);
            if (bi[d] >= B->nb[d]) bi[d] = B->nb[d] - 1;
            if (bi[d] < 0) bi[d] = 0;
        }
        bof[g] = bi[0] + B->nb[0] * (bi[1] + B->nb[1] * bi[2]);
        B->start[bof[g] + 1]++;
    }
    for (int b = 0; b < nbt; b++) B->start[b + 1] += B->start[b];
    for (int g = 0; g < n; g++) B->item[B->start[bof[g]] + fill[bof[g]]++] = g;
    free(bof);
    free(fill);
    return 0;
}

static void bucket_free(bucket_grid *B) { free(B->start); free(B->item); }

/* every centre whose bucket lies within `radius` of pt (periodic wrap),
 * each centre reported once */
static int bucket_query(const bucket_grid *B, const double *pt, double radius, const int *r, const int32_t *per,
                        int dim, int *out, int maxout)
{
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) {
        int span = (int)ceil(radius / B->bw[d]) + 1;
        int pb = (int)(pt[d] / B->bw[d]);
        if (2 * span + 1 >= B->nb[d]) { lo[d] = 0; hi[d] = B->nb[d] - 1; }
        else { lo[d] = pb - span; hi[d] = pb + span; }
        if (!per[d]) { if (lo[d] < 0) lo[d] = 0; if (hi[d] > B->nb[d] - 1) hi[d] = B->nb[d] - 1; }
    }
    int n = 0;
    for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
            for (int i = lo[0]; i <= hi[0]; i++) {
                int o[3] = {i, j, k}, bi[3];
                for (int d = 0; d < 3; d++) {
                    int v = o[d] % B->nb[d];
                    if (v < 0) v += B->nb[d];
                    bi[d] = v;
                }
                int b = bi[0] + B->nb[0] * (bi[1] + B->nb[1] * bi[2]);
                for (int t = B->start[b]; t < B->start[b + 1]; t++) {
                    if (n >= maxout) return n;
                    out[n++] = B->item[t];
                }
            }
    return n;
}

static void set_neighbours(long g, const int *r, const int32_t *per, int dim, long *nbs, int *nn)
{
    int x[3] = {(int)(g % r[0]), (int)((g / r[0]) % r[1]), (int)(g / ((long)r[0] * r[1]))};
    *nn = 0;
    for (int d = 0; d < dim; d++)
        for (int s = -1; s <= 1; s += 2) {
            int y[3] = {x[0], x[1], x[2]};
            y[d] += s;
            if (y[d] < 0 || y[d] >= r[d]) {
                if (!per[d]) continue;
                y[d] = (y[d] + r[d]) % r[d];
            }
            nbs[(*nn)++] = y[0] + (long)r[0] * (y[1] + (long)r[1] * y[2]);
        }
}

int cipher_initial_state_diffuse_aos(const cipher_problem *p, const cipher_mesh *m, double width, double *X)
{
    if (!p->centres || !p->voxelphase || width <= 0.0) return CIPHER_E_ARG;
    cipher_aos_layout L = cipher_problem_aos_layout(p);
    const int P = p->pf_size, dim = p->dim;
    int r[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) r[d] = p->resolution[d];
    const double pi = 3.14159265358979323846;
    long total = (long)r[0] * r[1] * r[2];
    uint16_t *own = (uint16_t *)malloc((size_t)total * (P + 1) * sizeof(uint16_t));
    double *ow = (double *)malloc((size_t)total * P * sizeof(double));
    unsigned char *bad = (unsigned char *)malloc((size_t)total);
    bucket_grid B;
    double cell_size = pow((double)total / p->npf, 1.0 / dim);
    if (!own || !ow || !bad || bucket_build(&B, p->centres, p->npf, r, dim, cell_size)) {
        free(own); free(ow); free(bad); bucket_free(&B);
        return CIPHER_E_NOMEM;
    }
    int cand[4096];
    /* own sets: the nearest grain (weight 1) and every grain whose bisector is
     * within width/2 (weight f/(1-f)); at most P, the largest weights kept */
    for (long g = 0; g < total; g++) {
        int x[3] = {(int)(g % r[0]), (int)((g / r[0]) % r[1]), (int)(g / ((long)r[0] * r[1]))};
        double pt[3] = {x[0] + 0.5, x[1] + 0.5, x[2] + 0.5};
        int oi = p->voxelphase[g];
        double vi[3] = {0, 0, 0}, di2 = 0.0;
        min_image(pt, &p->centres[3 * oi], r, p->periodic, dim, vi);
        for (int d = 0; d < dim; d++) di2 += vi[d] * vi[d];
        double lim = sqrt(di2) + width;
        int nq = bucket_query(&B, pt, lim, r, p->periodic, dim, cand, 4096);
        int cid[CIPHER_DIFFUSE_MAXCAND];
        double cw[CIPHER_DIFFUSE_MAXCAND];
        int nc = 0;
        cid[nc] = oi;
        cw[nc++] = 1.0;
        for (int q = 0; q < nq && nc < CIPHER_DIFFUSE_MAXCAND; q++) {
            int j = cand[q];
            if (j == oi) continue;
            int dup = 0;
            for (int a = 0; a < nc; a++) if (cid[a] == j) dup = 1;
            if (dup) continue;
            double vj[3] = {0, 0, 0}, dj2 = 0.0, dv2 = 0.0;
            min_image(pt, &p->centres[3 * j], r, p->periodic, dim, vj);
            for (int d = 0; d < dim; d++) dj2 += vj[d] * vj[d];
            if (dj2 > lim * lim) continue;
            for (int d = 0; d < dim; d++) dv2 += (vj[d] - vi[d]) * (vj[d] - vi[d]);
            if (dv2 <= 0.0) continue;
            double dist = (dj2 - di2) / (2.0 * sqrt(dv2));
            if (dist < 0.0) dist = 0.0;
            if (dist >= 0.5 * width) continue;
            double f = 0.5 - 0.5 * sin(pi * dist / width);
            cid[nc] = j;
            cw[nc++] = f / (1.0 - f);
        }
        /* largest weights first (owner stays first), cap at P */
        for (int a = 2; a < nc; a++)
            for (int b = a; b > 1 && cw[b] > cw[b - 1]; b--) {
                double tw = cw[b]; cw[b] = cw[b - 1]; cw[b - 1] = tw;
                int ti = cid[b]; cid[b] = cid[b - 1]; cid[b - 1] = ti;
            }
        if (nc > P) nc = P;
        uint16_t *o = &own[(size_t)g * (P + 1)];
        o[0] = (uint16_t)nc;
        for (int a = 0; a < nc; a++) { o[1 + a] = (uint16_t)cid[a]; ow[(size_t)g * P + a] = cw[a]; }
    }
    bucket_free(&B);
    /* repair: while a union with the neighbours exceeds P, drop the weakest
     * minority phase of that cell and of its neighbours */
    uint16_t set[CIPHER_MAXAP + 1], tmp[CIPHER_MAXAP + 1];
    long nbs[6];
    int nn;
    for (int iter = 0; iter < 64; iter++) {
        long nbad = 0;
        for (long g = 0; g < total; g++) {
            const uint16_t *o = &own[(size_t)g * (P + 1)];
            int n = o[0];
            memcpy(set, &o[1], (size_t)n * sizeof(uint16_t));
            for (int a = 1; a < n; a++)
                for (int b = a; b > 0 && set[b] < set[b - 1]; b--) { uint16_t t = set[b]; set[b] = set[b - 1]; set[b - 1] = t; }
            set_neighbours(g, r, p->periodic, dim, nbs, &nn);
            int over = 0;
            for (int k = 0; k < nn && !over; k++) {
                const uint16_t *q = &own[(size_t)nbs[k] * (P + 1)];
                uint16_t qs[CIPHER_MAXAP];
                int qn = q[0];
                memcpy(qs, &q[1], (size_t)qn * sizeof(uint16_t));
                for (int a = 1; a < qn; a++)
                    for (int b = a; b > 0 && qs[b] < qs[b - 1]; b--) { uint16_t t = qs[b]; qs[b] = qs[b - 1]; qs[b - 1] = t; }
                int u = set_union(tmp, set, n, qs, qn, P);
                if (u < 0) over = 1;
                else { memcpy(set, tmp, (size_t)u * sizeof(uint16_t)); n = u; }
            }
            bad[g] = (unsigned char)over;
            nbad += over;
        }
        if (!nbad) break;
        for (long g = 0; g < total; g++) {
            if (!bad[g]) continue;
            set_neighbours(g, r, p->periodic, dim, nbs, &nn);
            nbs[nn++] = g;
            for (int k = 0; k < nn; k++) {
                uint16_t *o = &own[(size_t)nbs[k] * (P + 1)];
                if (o[0] > 1) o[0]--;   /* the last entry has the smallest weight */
            }
        }
    }
    /* final state: own weights normalised, sets united with the neighbours' */
    memset(X, 0, (size_t)m->ncells * L.ndof * sizeof(double));
    int rc = 0;
    for (long lc = 0; lc < m->ncells && !rc; lc++) {
        long g = m->cell_global[lc];
        const uint16_t *o = &own[(size_t)g * (P + 1)];
        int n = o[0];
        double sum = 0.0;
        for (int a = 0; a < n; a++) sum += ow[(size_t)g * P + a];
        memcpy(set, &o[1], (size_t)n * sizeof(uint16_t));
        for (int a = 1; a < n; a++)
            for (int b = a; b > 0 && set[b] < set[b - 1]; b--) { uint16_t t = set[b]; set[b] = set[b - 1]; set[b - 1] = t; }
        set_neighbours(g, r, p->periodic, dim, nbs, &nn);
        for (int k = 0; k < nn; k++) {
            const uint16_t *q = &own[(size_t)nbs[k] * (P + 1)];
            uint16_t qs[CIPHER_MAXAP];
            int qn = q[0];
            memcpy(qs, &q[1], (size_t)qn * sizeof(uint16_t));
            for (int a = 1; a < qn; a++)
                for (int b = a; b > 0 && qs[b] < qs[b - 1]; b--) { uint16_t t = qs[b]; qs[b] = qs[b - 1]; qs[b - 1] = t; }
            int u = set_union(tmp, set, n, qs, qn, P);
            if (u < 0) { rc = CIPHER_E_CAP; break; }
            memcpy(set, tmp, (size_t)u * sizeof(uint16_t));
            n = u;
        }
        if (rc) break;
        double *cell = &X[lc * L.ndof];
        cell[L.as_offset] = (double)n;
        for (int a = 0; a < n; a++) {
            cell[L.as_offset + 1 + a] = (double)set[a];
            double v = 0.0;
            for (int k = 0; k < o[0]; k++)
                if (o[1 + k] == set[a]) v = ow[(size_t)g * P + k] / sum;
            cell[L.pf_offset + a] = v;
        }
        cell[L.tm_offset] = p->material[p->phasematerialmapping[p->voxelphase[g]]].temperature0;
    }
    free(own);
    free(ow);
    free(bad);
    return rc;
}

int cipher_abi_sizes(int64_t *out, int n)
{
    const int64_t s[12] = {(int64_t)sizeof(cipher_tseries), (int64_t)sizeof(cipher_rk), (int64_t)sizeof(cipher_mobility),
                           (int64_t)sizeof(cipher_source), (int64_t)sizeof(cipher_material),
                           (int64_t)sizeof(cipher_interface), (int64_t)sizeof(cipher_bc),
                           (int64_t)sizeof(cipher_problem), (int64_t)sizeof(cipher_mesh),
                           (int64_t)sizeof(cipher_nucleus), (int64_t)sizeof(cipher_output_field),
                           (int64_t)sizeof(cipher_config)};
    int k = n < 12 ? n : 12;
    for (int i = 0; i < k; i++) out[i] = s[i];
    return k;
}
