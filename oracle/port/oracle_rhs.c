/*
 * oracle_rhs.c - CPU restatement of CIPHER's RHSFunction (src/cipher.c:27-681),
 * the active-set part of PostStep (src/cipher.c:869-974) and SetUpProblem
 * (src/init.c:1721-1830) over the explicit mesh of cipher_problem.h.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * State vectors use the reference's per-cell AoS layout
 * [AS P+1 | PF P | DP D | EX P*S | TM 1] in doubles; Xlocal holds the owned
 * cells followed by the ghost cells of the mesh, F only the owned cells.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

#define OR_PI 3.14159265358979323846264338327950288419716939937510582

/* reference dof layout (init.c:1330-1343) */
static cipher_aos_layout or_layout(const cipher_problem *p)
{
    cipher_aos_layout L;
    int P = p->pf_size;
    L.sf_size = p->maxsites * p->ncp;
    L.sp_size = p->maxsites * p->ndp;
    L.as_offset = 0;
    L.as_size = P + 1;
    L.pf_offset = L.as_size;
    L.pf_size = P;
    L.dp_offset = L.pf_offset + P;
    L.dp_size = p->ndp;
    L.ex_offset = L.dp_offset + p->ndp;
    L.ex_size = P * L.sp_size;
    L.tm_offset = L.ex_offset + L.ex_size;
    L.ndof = L.tm_offset + 1;
    return L;
}

cipher_aos_layout or_aos_layout(const cipher_problem *p) { return or_layout(p); }

static void decode_set(const double *as, uint16_t *ids, int *n)
{
    *n = (int)round(as[0]);
    for (int k = 0; k < *n; k++) ids[k] = (uint16_t)round(as[1 + k]);
}

static const cipher_interface *pair_interface(const cipher_problem *p, int a, int b)
{
    return &p->interface[p->interfacelist[a * p->npf + b]];
}

/* solute source of one cell (material.c:295-351); random sources call rand()
 * in the reference and are not reproducible, so they are rejected upstream */
static void chem_source(const cipher_problem *p, const double *comp, const double *h,
                        const uint16_t *ids, int n, double *out)
{
    int ncp = p->ncp;
    double tmp[CIPHER_MAXCP];
    memset(out, 0, (size_t)ncp * sizeof(double));
    for (int k = 0; k < n; k++) {
        const cipher_material *m = or_material(p, ids[k]);
        for (int s = 0; s < m->nsources; s++) {
            for (int c = 0; c < ncp; c++) tmp[c] = m->sources[s].rate[c] * (m->sources[s].ceq[c] - comp[c]);
            for (int c = 0; c < ncp; c++) out[c] += h[k] * h[k] * tmp[c];
        }
        for (int j = k + 1; j < n; j++) {
            const cipher_interface *itf = pair_interface(p, ids[k], ids[j]);
            for (int s = 0; s < itf->nsources; s++) {
                for (int c = 0; c < ncp; c++) tmp[c] = itf->sources[s].rate[c] * (itf->sources[s].ceq[c] - comp[c]);
                for (int c = 0; c < ncp; c++) out[c] += 2.0 * h[k] * h[j] * tmp[c];
            }
        }
    }
}

static int check_supported(const cipher_problem *p, const cipher_mesh *m)
{
    if (p->gradient_calculation && !m->uniform) return 7;
    for (int m = 0; m < p->nmat; m++) {
        for (int s = 0; s < p->material[m].nsources; s++)
            if (p->material[m].sources[s].model != CIPHER_SOURCE_SINK) return 7;
        if (p->ndp == 0 && p->material[m].model != CIPHER_CHEM_NONE) return 7;
        if (p->ndp == 0 && p->material[m].tconductivity.n) return 7;
    }
    for (int i = 0; i < p->nf; i++)
        for (int s = 0; s < p->interface[i].nsources; s++)
            if (p->interface[i].sources[s].model != CIPHER_SOURCE_SINK) return 7;
    return 0;
}

/* phase-field gradients of the owned cells (src/cipher.c:82-146) with the
 * least-squares weights of src/cipher.c:1232-1282: each owned cell's face
 * neighbours in face order, centroid offsets ((i + 0.5) * size / resolution
 * per axis of the grid index, raw across periodic sides), AtA, its inverse,
 * (AtA)^-1 At; grad[(c*dim + d)*P + g] */
static int gradients(const cipher_problem *p, const cipher_mesh *m, const double *X, const cipher_aos_layout *L,
                     double *grad)
{
    const int dim = p->dim, P = p->pf_size, ndof = L->ndof;
    const int nown = m->nowned;
    int *cnt = (int *)calloc((size_t)nown, sizeof(int));
    int *nbr = (int *)malloc((size_t)nown * 24 * sizeof(int));
    if (!cnt || !nbr) { free(cnt); free(nbr); return 2; }
    for (int f = 0; f < m->nfaces; f++) {
        const int a = m->face_cells[2 * f], b = m->face_cells[2 * f + 1];
        if (a == b) continue;
        if (a < nown && cnt[a] < 24) nbr[a * 24 + cnt[a]++] = b;
        if (b < nown && cnt[b] < 24) nbr[b * 24 + cnt[b]++] = a;
    }
    uint16_t ids[CIPHER_MAXAP], nids[CIPHER_MAXAP];
    for (int c = 0; c < nown; c++) {
        double xc[3], A[24 * 3], ata[9], inv[9], w[3 * 24];
        const int nls = cnt[c];
        int64_t g = m->cell_global[c];
        for (int d = 0; d < dim; d++) {
            xc[d] = ((double)(g % p->resolution[d]) + 0.5) * (p->size[d] / p->resolution[d]);
            g /= p->resolution[d];
        }
        for (int k = 0; k < nls; k++) {
            int64_t q = m->cell_global[nbr[c * 24 + k]];
            for (int d = 0; d < dim; d++) {
                A[k * dim + d] = ((double)(q % p->resolution[d]) + 0.5) * (p->size[d] / p->resolution[d]);
                q /= p->resolution[d];
                A[k * dim + d] -= xc[d];
            }
        }
        for (int i = 0; i < dim; i++)
            for (int j = i; j < dim; j++) {
                double v = 0.0;
                for (int k = 0; k < nls; k++) v += A[k * dim + i] * A[k * dim + j];
                ata[i * dim + j] = v;
                ata[j * dim + i] = v;
            }
        or_invert(inv, ata, dim);
        for (int i = 0; i < dim; i++)
            for (int k = 0; k < nls; k++) {
                double v = 0.0;
                for (int d = 0; d < dim; d++) v += inv[i * dim + d] * A[k * dim + d];
                w[i * nls + k] = v;
            }
        const double *cell = &X[(size_t)c * ndof];
        int n;
        decode_set(&cell[L->as_offset], ids, &n);
        const double *phi = &cell[L->pf_offset];
        double *gc = &grad[(size_t)c * dim * P];
        for (int q = 0; q < dim * P; q++) gc[q] = 0.0;
        for (int s = 0; s < n; s++)
            for (int d = 0; d < dim; d++) {
                double v = 0.0;
                for (int k = 0; k < nls; k++) v -= w[d * nls + k] * phi[s];
                gc[d * P + s] = v;
            }
        for (int k = 0; k < nls; k++) {
            const double *nc = &X[(size_t)nbr[c * 24 + k] * ndof];
            int nn;
            decode_set(&nc[L->as_offset], nids, &nn);
            for (int i = 0, j = 0; i < n && j < nn;) {
                if (ids[i] == nids[j]) {
                    for (int d = 0; d < dim; d++) gc[d * P + i] += w[d * nls + k] * nc[L->pf_offset + j];
                    i++;
                    j++;
                } else if (ids[i] < nids[j]) i++;
                else j++;
            }
        }
    }
    free(cnt);
    free(nbr);
    return 0;
}

int oracle_rhs(const cipher_problem *p, const cipher_mesh *m, double t, const double *X, double *F)
{
    (void)t;
    int rc = check_supported(p, m);
    if (rc) return rc;
    cipher_aos_layout L = or_layout(p);
    const int ndof = L.ndof, P = p->pf_size, ncp = p->ncp, ndp = p->ndp;
    const int SP = L.sp_size, SF = L.sf_size, dim = p->dim;
    const int ncells = m->ncells, nowned = m->nowned;
    const int interp = p->interpolation;

    memset(F, 0, (size_t)nowned * ndof * sizeof(double));
    double *lap = (double *)calloc((size_t)ncells * ndof, sizeof(double));
    double *yall = (double *)calloc((size_t)ncells * P * (SF > 0 ? SF : 1), sizeof(double));
    double *comp = (double *)calloc((size_t)ncells * ncp, sizeof(double));
    double *mob = (double *)calloc((size_t)ncells * ncp, sizeof(double));
    double *tcond = (double *)calloc((size_t)ncells, sizeof(double));
    if (!lap || !yall || !comp || !mob || !tcond) { free(lap); free(yall); free(comp); free(mob); free(tcond); return 2; }

    uint16_t ids[CIPHER_MAXAP], idsL[CIPHER_MAXAP], idsR[CIPHER_MAXAP];
    uint16_t com[CIPHER_MAXAP], inL[CIPHER_MAXAP], inR[CIPHER_MAXAP];
    double h[CIPHER_MAXAP], pot[2 * CIPHER_MAXCP], melem[CIPHER_MAXCP], ci[CIPHER_MAXCP];
    int n, nL, nR;

    /* ---- per-cell site fractions, composition, mobility (cipher.c:148-233) ---- */
    for (int c = 0; c < ncells; c++) {
        const double *cell = &X[(size_t)c * ndof];
        decode_set(&cell[L.as_offset], ids, &n);
        const double *phi = &cell[L.pf_offset];
        const double *mu = &cell[L.dp_offset];
        const double *ex = &cell[L.ex_offset];
        double T = cell[L.tm_offset];
        or_interpolant(interp, phi, n, h);
        if (ndp) {
            double *y = &yall[(size_t)c * P * SF];
            double *cc = &comp[(size_t)c * ncp], *mm = &mob[(size_t)c * ncp];
            memset(ci, 0, sizeof(ci));
            for (int k = 0; k < n; k++)
                for (int j = k + 1; j < n; j++) {
                    const cipher_interface *itf = pair_interface(p, ids[k], ids[j]);
                    if (itf->has_potential)
                        for (int d = 0; d < ndp; d++) ci[d] += h[k] * h[j] * itf->potential[d];
                }
            tcond[c] = 0.0;
            for (int g = 0; g < n; g++) {
                const cipher_material *mat = or_material(p, ids[g]);
                for (int s = 0; s < mat->nsites; s++)
                    for (int d = 0; d < ndp; d++)
                        pot[s * ndp + d] = mat->stoichiometry[s] * (mu[d] - ci[d]) - ex[g * SP + s * ndp + d];
                or_sitefrac(p, ids[g], pot, T, &y[g * SF]);
                or_mobility(p, ids[g], &y[g * SF], T, melem);
                for (int d = 0; d < ncp; d++) mm[d] += h[g] * melem[d];
                for (int s = 0; s < mat->nsites; s++)
                    for (int d = 0; d < ncp; d++) cc[d] += h[g] * mat->stoichiometry[s] * y[g * SF + s * ncp + d];
                if (mat->tconductivity.n) tcond[c] += h[g] * or_tseries(T, &mat->tconductivity);
            }
            for (int k = 0; k < n; k++)
                for (int j = k + 1; j < n; j++) {
                    const cipher_interface *itf = pair_interface(p, ids[k], ids[j]);
                    if (itf->has_mobilityc)
                        for (int d = 0; d < ncp; d++) mm[d] *= exp(itf->mobilityc[d] / CIPHER_R_GAS / T);
                }
        } else {
            tcond[c] = 0.0;   /* no conductivity allowed without chemistry (checked above) */
        }
    }

    /* ---- face fluxes in face order (cipher.c:235-317) ---- */
    for (int f = 0; f < m->nfaces; f++) {
        int cl = m->face_cells[2 * f], cr = m->face_cells[2 * f + 1];
        if (cl >= ncells || cr >= ncells) continue;
        const double *xl = &X[(size_t)cl * ndof], *xr = &X[(size_t)cr * ndof];
        double *ll = &lap[(size_t)cl * ndof], *lr = &lap[(size_t)cr * ndof];
        decode_set(&xl[L.as_offset], idsL, &nL);
        decode_set(&xr[L.as_offset], idsR, &nR);
        double dl = m->cellgeom[cl], dr = m->cellgeom[cr];
        double vl = or_ipow(dl, (unsigned)dim), vr = or_ipow(dr, (unsigned)dim);
        double ff = 2.0 * (dl < dr ? vl / dl : vr / dr) / (dl + dr);
        /* the reference gates the phase flux on the L cell only (cipher.c:277) */
        if (nL > 1 || idsL[0] > 1) {
            int nc = or_set_intersect(idsL, nL, idsR, nR, com, inL, inR);
            for (int k = 0; k < nc; k++) {
                double flux = xr[L.pf_offset + inR[k]] - xl[L.pf_offset + inL[k]];
                ll[L.pf_offset + inL[k]] += ff * flux / vl;
                lr[L.pf_offset + inR[k]] -= ff * flux / vr;
            }
        }
        if (ndp) {
            double me[CIPHER_MAXCP], ca[CIPHER_MAXCP], MB[CIPHER_MAXCP * CIPHER_MAXCP], dmu[CIPHER_MAXCP], fl[CIPHER_MAXCP];
            const double *ml = &mob[(size_t)cl * ncp], *mr = &mob[(size_t)cr * ncp];
            const double *cL = &comp[(size_t)cl * ncp], *cR = &comp[(size_t)cr * ncp];
            for (int d = 0; d < ncp; d++) {
                if (fabs(ml[d]) > 1e-32 && fabs(mr[d]) > 1e-32) me[d] = 2.0 * ml[d] * mr[d] / (ml[d] + mr[d]);
                else me[d] = 0.0;
                ca[d] = 2.0 * cL[d] * cR[d] / (cL[d] + cR[d]);
            }
            /* Andersson-Agren volume-fixed frame (material.c:1125-1137) */
            for (int i = 0; i < ndp; i++)
                for (int j = 0; j < ndp; j++) {
                    double acc = 0.0;
                    for (int k = 0; k < ncp; k++)
                        acc += ((j == k ? 1.0 : 0.0) - ca[j]) * ((k == i ? 1.0 : 0.0) - ca[i]) * me[k];
                    MB[i * ndp + j] = acc;
                }
            for (int d = 0; d < ndp; d++) dmu[d] = xr[L.dp_offset + d] - xl[L.dp_offset + d];
            or_matvec(fl, MB, dmu, ndp);
            for (int d = 0; d < ndp; d++) {
                ll[L.dp_offset + d] += ff * fl[d] / vl;
                lr[L.dp_offset + d] -= ff * fl[d] / vr;
            }
        }
        if (fabs(tcond[cl]) > 1e-32 && fabs(tcond[cr]) > 1e-32) {
            double ft = 2.0 * tcond[cl] * tcond[cr] / (tcond[cl] + tcond[cr])
                      * (xr[L.tm_offset] - xl[L.tm_offset]);
            ll[L.tm_offset] += ff * ft / vl;
            lr[L.tm_offset] -= ff * ft / vr;
        }
    }

    /* ---- boundary faces (cipher.c:319-389) ---- */
    {
        double fluxt = 0.0;
        for (int b = 0; b < p->nbcs; b++) {
            const cipher_bc *bc = &p->bcs[b];
            for (int k = 0; k < m->nbfaces; k++) {
                if (m->bface_label[k] != bc->boundaryid) continue;
                int c = m->bface_cell[k];
                const double *xc = &X[(size_t)c * ndof];
                double dc = m->cellgeom[c];
                double fd[CIPHER_MAXCP] = {0};
                if (bc->chem_bctype != CIPHER_BC_NONE) {
                    if (bc->chem_bctype == CIPHER_BC_NEUMANN) {
                        for (int d = 0; d < ndp; d++) if (bc->chem_bcbool[d]) fd[d] = bc->chem_bcval[d] * dc;
                    } else {
                        for (int d = 0; d < ndp; d++)
                            if (bc->chem_bcbool[d]) fd[d] = mob[(size_t)c * ncp + d] * (bc->chem_bcval[d] - xc[L.dp_offset + d]);
                    }
                }
                if (bc->thermal_bctype == CIPHER_BC_NEUMANN) fluxt = tcond[c] * bc->thermal_bcval * dc;
                else if (bc->thermal_bctype == CIPHER_BC_DIRICHLET) fluxt = tcond[c] * (bc->thermal_bcval - xc[L.tm_offset]);
                double *lc = &lap[(size_t)c * ndof];
                double cf = 1.0 / or_ipow(dc, 2);
                if (bc->chem_bctype != CIPHER_BC_NONE)
                    for (int d = 0; d < ndp; d++) lc[L.dp_offset + d] += cf * fd[d];
                if (bc->thermal_bctype != CIPHER_BC_NONE) lc[L.tm_offset] += cf * fluxt;
            }
        }
    }

    /* ---- gradients for anisotropic interfaces (cipher.c:82-146) ---- */
    double *grad = NULL;
    int aniso = 0;
    for (int i = 0; p->gradient_calculation && i < p->nf; i++)
        if (p->interface[i].energy_naniso > 0 || p->interface[i].mobility_naniso > 0) aniso = 1;
    if (aniso) {
        grad = (double *)malloc((size_t)nowned * dim * P * sizeof(double));
        if (!grad || gradients(p, m, X, &L, grad)) {
            free(grad); free(lap); free(yall); free(comp); free(mob); free(tcond);
            return 2;
        }
    }

    /* ---- per owned cell (cipher.c:391-664) ---- */
    for (int c = 0; c < nowned; c++) {
        const double *cell = &X[(size_t)c * ndof];
        const double *lc = &lap[(size_t)c * ndof];
        double *fc = &F[(size_t)c * ndof];
        decode_set(&cell[L.as_offset], ids, &n);
        const double *phi = &cell[L.pf_offset];
        const double *mu = &cell[L.dp_offset];
        const double *ex = &cell[L.ex_offset];
        double T = cell[L.tm_offset];
        const double *plap = &lc[L.pf_offset];
        const double *y = &yall[(size_t)c * P * SF];
        double *pf = &fc[L.pf_offset];
        or_interpolant(interp, phi, n, h);

        if (n > 1) {
            double sig[CIPHER_MAXAP * CIPHER_MAXAP], mij[CIPHER_MAXAP * CIPHER_MAXAP], wid[CIPHER_MAXAP * CIPHER_MAXAP];
            double cap[CIPHER_MAXAP], chem[CIPHER_MAXAP], unc[CIPHER_MAXAP];
            int act[CIPHER_MAXAP];
            for (int k = 0; k < n; k++)
                for (int j = k + 1; j < n; j++) {
                    const cipher_interface *itf = pair_interface(p, ids[k], ids[j]);
                    int kj = k * n + j;
                    sig[kj] = 1.0;
                    mij[kj] = 1.0;
                    if (grad) {   /* anisotropy about the pair's normal (cipher.c:427-460) */
                        const double *gc = &grad[(size_t)c * dim * P];
                        double u[3], nrm = 0.0;
                        for (int d = 0; d < dim; d++) {
                            u[d] = gc[d * P + k] - gc[d * P + j];
                            nrm += u[d] * u[d];
                        }
                        nrm = sqrt(nrm);
                        if (nrm > 1e-16)
                            for (int d = 0; d < dim; d++) u[d] /= nrm;
                        for (int q = 0; q < itf->energy_naniso; q++) {
                            double dot = 0.0;
                            for (int d = 0; d < dim; d++) dot += u[d] * itf->energy_aniso_dir[dim * q + d];
                            sig[kj] += or_ipow(dot, 4) * itf->energy_aniso_val[q];
                        }
                        for (int q = 0; q < itf->mobility_naniso; q++) {
                            double dot = 0.0;
                            for (int d = 0; d < dim; d++) dot += u[d] * itf->mobility_aniso_dir[dim * q + d];
                            mij[kj] += or_ipow(dot, 4) * itf->mobility_aniso_val[q];
                        }
                    }
                    sig[kj] *= itf->energy_m0;
                    if (itf->energy_activation.n)
                        sig[kj] *= exp(or_tseries(T, &itf->energy_activation) / CIPHER_R_GAS / T);
                    mij[kj] *= itf->mobility_m0;
                    if (itf->mobility_activation.n)
                        mij[kj] *= exp(or_tseries(T, &itf->mobility_activation) / CIPHER_R_GAS / T);
                    wid[kj] = itf->width;
                }
            /* capillary force with triple-junction penalty (cipher.c:474-497) */
            memset(cap, 0, sizeof(cap));
            for (int k = 0; k < n; k++) {
                for (int j = k + 1; j < n; j++) {
                    int kj = k * n + j;
                    cap[k] -= sig[kj] * (phi[j] / wid[kj] + plap[j] * wid[kj] / OR_PI / OR_PI);
                    cap[j] -= sig[kj] * (phi[k] / wid[kj] + plap[k] * wid[kj] / OR_PI / OR_PI);
                    for (int i = j + 1; i < n; i++) {
                        double tj = 0.0, v;
                        v = sig[k * n + j] / wid[k * n + j]; tj = tj > v ? tj : v;
                        v = sig[k * n + i] / wid[k * n + i]; tj = tj > v ? tj : v;
                        v = sig[j * n + i] / wid[j * n + i]; tj = tj > v ? tj : v;
                        tj *= p->junctionpenalty;
                        cap[k] -= tj * phi[j] * phi[i];
                        cap[j] -= tj * phi[k] * phi[i];
                        cap[i] -= tj * phi[k] * phi[j];
                    }
                }
                cap[k] *= 8.0;
                cap[k] += plap[k];
            }
            /* chemical driving force (cipher.c:499-522) */
            double cbar[CIPHER_MAXCP] = {0};
            for (int g = 0; g < n; g++) chem[g] = or_chemenergy(p, ids[g], &y[g * SF], mu, T);
            for (int g = 0; g < n; g++) {
                const cipher_material *mat = or_material(p, ids[g]);
                for (int s = 0; s < mat->nsites; s++)
                    for (int d = 0; d < ndp; d++) cbar[d] += h[g] * mat->stoichiometry[s] * y[g * SF + s * ncp + d];
            }
            for (int k = 0; k < n; k++)
                for (int j = k + 1; j < n; j++) {
                    const cipher_interface *itf = pair_interface(p, ids[k], ids[j]);
                    if (itf->has_potential) {
                        double v = 0.0;
                        for (int d = 0; d < ndp; d++) v += itf->potential[d] * cbar[d];
                        chem[k] += v * h[j];
                        chem[j] += v * h[k];
                    }
                }
            or_interpolant_dT(interp, chem, phi, n);
            /* active set and constrained rate (cipher.c:524-555) */
            double nact = 0.0;
            memset(unc, 0, sizeof(unc));
            for (int k = 0; k < n; k++) {
                for (int j = k + 1; j < n; j++) {
                    int kj = k * n + j;
                    double r = mij[kj] * ((cap[k] - cap[j]) - (chem[k] - chem[j]) * 8.0 * sqrt(h[k] * h[j]) / OR_PI);
                    unc[k] += r;
                    unc[j] -= r;
                }
                act[k] = (phi[k] > CIPHER_TOL && phi[k] < 1.0 - CIPHER_TOL)
                      || (phi[k] < CIPHER_TOL && unc[k] > 0.0)
                      || (phi[k] > 1.0 - CIPHER_TOL && unc[k] < 0.0);
                if (act[k]) nact += 1.0;
            }
            for (int k = 0; k < n; k++) {
                if (!act[k]) continue;
                for (int j = k + 1; j < n; j++) {
                    if (!act[j]) continue;
                    int kj = k * n + j;
                    double r = mij[kj] * ((cap[k] - cap[j]) - (chem[k] - chem[j]) * 8.0 * sqrt(h[k] * h[j]) / OR_PI);
                    pf[k] += r;
                    pf[j] -= r;
                }
                pf[k] /= nact;
            }
        }

        /* temperature rate (cipher.c:558-568) */
        double cp = 0.0, tr = lc[L.tm_offset];
        for (int g = 0; g < n; g++) {
            const cipher_material *mat = or_material(p, ids[g]);
            if (mat->specific_heat.n) cp += h[g] * or_tseries(T, &mat->specific_heat);
            if (mat->latent_heat.n) tr += pf[g] * or_tseries(T, &mat->latent_heat);
        }
        if (cp != 0.0) tr /= cp;
        if (p->has_temperature_rate) tr += p->temperature_rate[p->currentloadcase];
        fc[L.tm_offset] = tr;

        if (ndp) {
            double *dex = &fc[L.ex_offset];
            double spx[2 * CIPHER_MAXCP];
            /* explicit potential relaxation (cipher.c:570-581) */
            for (int g = 0; g < n; g++) {
                const cipher_material *mat = or_material(p, ids[g]);
                or_sitepot_explicit(p, ids[g], &y[g * SF], T, spx);
                for (int s = 0; s < mat->nsites; s++)
                    for (int d = 0; d < ndp; d++)
                        dex[g * SP + s * ndp + d] = mat->chempot_ex_kineticcoeff * (spx[s * ndp + d] - ex[g * SP + s * ndp + d]);
            }
            /* composition rate and dmu/dt (cipher.c:583-662) */
            double cpv[CIPHER_MAXAP * CIPHER_MAXCP];
            double tpot[CIPHER_MAXAP * 2 * CIPHER_MAXCP * CIPHER_MAXCP], tex[CIPHER_MAXAP * 2 * CIPHER_MAXCP * CIPHER_MAXCP];
            double tT[CIPHER_MAXAP * 2 * CIPHER_MAXCP];
            double dcdm[CIPHER_MAXCP * CIPHER_MAXCP], dmdc[CIPHER_MAXCP * CIPHER_MAXCP];
            double wdp[CIPHER_MAXCP], tmp[CIPHER_MAXCP], wpf[CIPHER_MAXAP], src[CIPHER_MAXCP];
            const int DPn = ndp;
            memset(ci, 0, sizeof(ci));
            memset(cpv, 0, sizeof(cpv));
            for (int k = 0; k < n; k++)
                for (int j = k + 1; j < n; j++) {
                    const cipher_interface *itf = pair_interface(p, ids[k], ids[j]);
                    if (itf->has_potential)
                        for (int d = 0; d < ndp; d++) {
                            ci[d] += h[k] * h[j] * itf->potential[d];
                            cpv[k * DPn + d] += itf->potential[d] * h[j];
                            cpv[j * DPn + d] += itf->potential[d] * h[k];
                        }
                }
            memset(dcdm, 0, sizeof(dcdm));
            for (int g = 0; g < n; g++) {
                const cipher_material *mat = or_material(p, ids[g]);
                for (int s = 0; s < mat->nsites; s++)
                    for (int d = 0; d < ndp; d++)
                        pot[s * ndp + d] = mat->stoichiometry[s] * (mu[d] - ci[d]) - ex[g * SP + s * ndp + d];
                or_sitefrac_tangent(p, ids[g], &y[g * SF], pot, T,
                                    &tpot[g * SP * DPn], &tex[g * SP * DPn], &tT[g * SP]);
                for (int s = 0; s < mat->nsites; s++)
                    for (int q = 0; q < ndp * ndp; q++)
                        dcdm[q] += h[g] * mat->stoichiometry[s] * mat->stoichiometry[s] * tpot[g * SP * DPn + s * DPn * DPn + q];
            }
            for (int g = 0; g < n; g++) {
                memcpy(tmp, &cpv[g * DPn], (size_t)DPn * sizeof(double));
                or_matvec(&cpv[g * DPn], dcdm, tmp, DPn);
            }
            memset(wdp, 0, sizeof(wdp));
            if (n > 1) {
                for (int d = 0; d < ndp; d++) {
                    for (int g = 0; g < n; g++) {
                        const cipher_material *mat = or_material(p, ids[g]);
                        wpf[g] = 0.0;
                        for (int s = 0; s < mat->nsites; s++) wpf[g] += mat->stoichiometry[s] * y[g * SF + s * ncp + d];
                        wpf[g] -= cpv[g * DPn + d];
                    }
                    or_interpolant_dT(interp, wpf, phi, n);
                    for (int g = 0; g < n; g++) wdp[d] -= pf[g] * wpf[g];
                }
            }
            chem_source(p, &comp[(size_t)c * ncp], h, ids, n, src);
            for (int d = 0; d < ndp; d++) wdp[d] += (lc[L.dp_offset + d] + src[d]);
            for (int g = 0; g < n; g++) {
                const cipher_material *mat = or_material(p, ids[g]);
                for (int s = 0; s < mat->nsites; s++) {
                    or_matvec(&cpv[g * DPn], &tex[g * SP * DPn + s * DPn * DPn], &dex[g * SP + s * DPn], DPn);
                    for (int d = 0; d < ndp; d++)
                        wdp[d] -= h[g] * mat->stoichiometry[s] * (cpv[g * DPn + d] + tT[g * SP + s * DPn + d] * tr);
                }
            }
            or_invert(dmdc, dcdm, DPn);
            or_matvec(&fc[L.dp_offset], dmdc, wdp, DPn);
        }
    }
    free(grad); free(lap); free(yall); free(comp); free(mob); free(tcond);
    return 0;
}

/* neighbour lists from the face table (any order: unions commute) */
static int build_neighbours(const cipher_mesh *m, int **off_out, int **nb_out)
{
    int *off = (int *)calloc((size_t)m->ncells + 1, sizeof(int));
    int *nb = (int *)malloc((size_t)(2 * m->nfaces + 1) * sizeof(int));
    if (!off || !nb) { free(off); free(nb); return 2; }
    for (int f = 0; f < m->nfaces; f++) {
        off[m->face_cells[2 * f] + 1]++;
        off[m->face_cells[2 * f + 1] + 1]++;
    }
    for (int c = 0; c < m->ncells; c++) off[c + 1] += off[c];
    int *fill = (int *)calloc((size_t)m->ncells, sizeof(int));
    for (int f = 0; f < m->nfaces; f++) {
        int a = m->face_cells[2 * f], b = m->face_cells[2 * f + 1];
        nb[off[a] + fill[a]++] = b;
        nb[off[b] + fill[b]++] = a;
    }
    free(fill);
    *off_out = off;
    *nb_out = nb;
    return 0;
}

/* active-set update (cipher.c:869-974): returns 3 when a superset exceeds P */
int oracle_poststep(const cipher_problem *p, const cipher_mesh *m, double *X)
{
    if (m->ncells != m->nowned) return 1;
    cipher_aos_layout L = or_layout(p);
    const int ndof = L.ndof, P = p->pf_size, SP = L.sp_size, ncells = m->ncells;
    uint16_t *pruned = (uint16_t *)malloc((size_t)ncells * (P + 1) * sizeof(uint16_t));
    int *off = NULL, *nbl = NULL;
    if (!pruned || build_neighbours(m, &off, &nbl)) { free(pruned); return 2; }
    uint16_t ids[CIPHER_MAXAP];
    int n;
    /* projection and pruning */
    for (int c = 0; c < ncells; c++) {
        double *cell = &X[(size_t)c * ndof];
        decode_set(&cell[L.as_offset], ids, &n);
        double *phi = &cell[L.pf_offset];
        uint16_t *pr = &pruned[(size_t)c * (P + 1)];
        if (n > 1) {
            double up[CIPHER_MAXAP];
            memcpy(up, phi, (size_t)n * sizeof(double));
            or_simplex_projection(phi, up, n);
            pr[0] = 0;
            for (int g = 0; g < n; g++) if (phi[g] > CIPHER_TOL) pr[1 + pr[0]++] = ids[g];
        } else {
            phi[0] = 1.0;
            pr[0] = 1;
            pr[1] = ids[0];
        }
    }
    /* union with neighbours and reorder */
    int rc = 0;
    for (int c = 0; c < ncells; c++) {
        double *cell = &X[(size_t)c * ndof];
        decode_set(&cell[L.as_offset], ids, &n);
        double *phi = &cell[L.pf_offset];
        double *ex = &cell[L.ex_offset];
        double T = cell[L.tm_offset];
        uint16_t sup[CIPHER_MAXAP + 1], tmp[CIPHER_MAXAP + 1];
        const uint16_t *own = &pruned[(size_t)c * (P + 1)];
        int ns = own[0];
        memcpy(sup, &own[1], (size_t)ns * sizeof(uint16_t));
        for (int k = off[c]; k < off[c + 1]; k++) {
            int nb = nbl[k];
            if (nb == c) continue;
            const uint16_t *o = &pruned[(size_t)nb * (P + 1)];
            int nn = or_set_union(sup, ns, &o[1], o[0], tmp, P);
            if (nn > P) { rc = 3; ns = P; break; }
            memcpy(sup, tmp, (size_t)nn * sizeof(uint16_t));
            ns = nn;
        }
        if (rc) break;
        double phiss[CIPHER_MAXAP], exss[CIPHER_MAXAP * 2 * CIPHER_MAXCP];
        for (int g = 0; g < ns; g++) {
            phiss[g] = 0.0;
            if (SP) or_sitepot_explicit(p, sup[g], or_material(p, sup[g])->c0, T, &exss[g * SP]);
        }
        uint16_t com[CIPHER_MAXAP], ia[CIPHER_MAXAP], ib[CIPHER_MAXAP];
        int nc = or_set_intersect(ids, n, sup, ns, com, ia, ib);
        for (int g = 0; g < nc; g++) {
            phiss[ib[g]] = phi[ia[g]];
            memcpy(&exss[ib[g] * SP], &ex[ia[g] * SP], (size_t)SP * sizeof(double));
        }
        memcpy(phi, phiss, (size_t)ns * sizeof(double));
        memcpy(ex, exss, (size_t)ns * SP * sizeof(double));
        cell[L.as_offset] = (double)ns;
        for (int g = 0; g < ns; g++) cell[L.as_offset + 1 + g] = (double)sup[g];
    }
    free(pruned); free(off); free(nbl);
    return rc;
}

/* initial state (init.c:1721-1830) for a whole-domain mesh */
int oracle_initial_state(const cipher_problem *p, const cipher_mesh *m, double *X)
{
    if (m->ncells != m->nowned || !p->voxelphase) return 1;
    cipher_aos_layout L = or_layout(p);
    const int ndof = L.ndof, P = p->pf_size, SP = L.sp_size, ndp = p->ndp;
    int *off = NULL, *nbl = NULL;
    if (build_neighbours(m, &off, &nbl)) return 2;
    memset(X, 0, (size_t)m->ncells * ndof * sizeof(double));
    int rc = 0;
    for (int c = 0; c < m->ncells && !rc; c++) {
        int own = p->voxelphase[m->cell_global[c]];
        uint16_t set[CIPHER_MAXAP + 1], tmp[CIPHER_MAXAP + 1], one[1];
        int n = 1;
        set[0] = (uint16_t)own;
        for (int k = off[c]; k < off[c + 1]; k++) {
            int nb = nbl[k];
            if (nb == c) continue;
            one[0] = (uint16_t)p->voxelphase[m->cell_global[nb]];
            int nn = or_set_union(set, n, one, 1, tmp, P);
            if (nn > P) { rc = 3; break; }
            memcpy(set, tmp, (size_t)nn * sizeof(uint16_t));
            n = nn;
        }
        double *cell = &X[(size_t)c * ndof];
        cell[L.as_offset] = (double)n;
        for (int g = 0; g < n; g++) cell[L.as_offset + 1 + g] = (double)set[g];
        double T = 0.0;
        for (int g = 0; g < n; g++) if (set[g] == own) T = or_material(p, own)->temperature0;
        cell[L.tm_offset] = T;
        for (int g = 0; g < n; g++) {
            const cipher_material *mat = or_material(p, set[g]);
            if (SP) or_sitepot_explicit(p, set[g], mat->c0, T, &cell[L.ex_offset + g * SP]);
            if (set[g] == own) {
                double sp[2 * CIPHER_MAXCP];
                cell[L.pf_offset + g] = 1.0;
                if (ndp) {
                    or_sitepot_total(p, set[g], mat->c0, T, sp);
                    for (int d = 0; d < ndp; d++) cell[L.dp_offset + d] = 0.0;
                    for (int s = 0; s < mat->nsites; s++)
                        for (int d = 0; d < ndp; d++) cell[L.dp_offset + d] += sp[s * ndp + d];
                }
            } else {
                cell[L.pf_offset + g] = 0.0;
            }
        }
    }
    free(off); free(nbl);
    return rc;
}

/* derived output fields (cipher.c:990-1078) of the owned cells:
 * out[k*nowned + c]; kinds/idx as the library's CIPHER_OUT_* descriptors */
int oracle_output_fields(const cipher_problem *p, const cipher_mesh *m, const double *X, const int32_t *kinds,
                         const int32_t *idx, int nf, double *out)
{
    cipher_aos_layout L = or_layout(p);
    const int ndof = L.ndof, ncp = p->ncp, ndp = p->ndp, SP = L.sp_size, SF = L.sf_size;
    uint16_t ids[CIPHER_MAXAP];
    double h[CIPHER_MAXAP], pot[2 * CIPHER_MAXCP], y[CIPHER_MAXAP * 2 * CIPHER_MAXCP];
    int n;
    (void)SF;
    for (int c = 0; c < m->nowned; c++) {
        const double *cell = &X[(size_t)c * ndof];
        decode_set(&cell[L.as_offset], ids, &n);
        const double *phi = &cell[L.pf_offset];
        const double *mu = &cell[L.dp_offset];
        const double *ex = &cell[L.ex_offset];
        double T = cell[L.tm_offset];
        or_interpolant(p->interpolation, phi, n, h);
        for (int k = 0; k < nf; k++) {
            double v = 0.0, mx;
            switch (kinds[k]) {
            case 0: case 1:
                mx = -CIPHER_LARGE;
                for (int g = 0; g < n; g++)
                    if (h[g] > mx) { mx = h[g]; v = kinds[k] == 0 ? (double)ids[g] : (double)p->phasematerialmapping[ids[g]]; }
                break;
            case 2:
                v = -1.0;
                for (int a = 0; a < n; a++)
                    for (int b = a + 1; b < n; b++) v = (double)p->interfacelist[ids[a] * p->npf + ids[b]];
                break;
            case 3:
                v = (idx[k] >= 0 && idx[k] < ndp) ? mu[idx[k]] : 0.0;
                break;
            case 4: {
                double ci[CIPHER_MAXCP] = {0}, avg[CIPHER_MAXCP] = {0};
                if (ndp) {
                    for (int a = 0; a < n; a++)
                        for (int b = a + 1; b < n; b++) {
                            const cipher_interface *itf = pair_interface(p, ids[a], ids[b]);
                            if (itf->has_potential)
                                for (int d = 0; d < ndp; d++) ci[d] += h[a] * h[b] * itf->potential[d];
                        }
                    for (int g = 0; g < n; g++) {
                        const cipher_material *mat = or_material(p, ids[g]);
                        for (int s = 0; s < mat->nsites; s++)
                            for (int d = 0; d < ndp; d++)
                                pot[s * ndp + d] = mat->stoichiometry[s] * (mu[d] - ci[d]) - ex[g * SP + s * ndp + d];
                        or_sitefrac(p, ids[g], pot, T, y);
                        for (int s = 0; s < mat->nsites; s++)
                            for (int d = 0; d < ncp; d++) avg[d] += h[g] * mat->stoichiometry[s] * y[s * ncp + d];
                    }
                }
                v = (idx[k] >= 0 && idx[k] < ncp) ? avg[idx[k]] : 0.0;
                break;
            }
            case 5:
                for (int g = 0; g < n; g++)
                    if ((int)ids[g] == idx[k]) v = phi[g];
                break;
            case 6:
                v = T;
                break;
            default:
                return 1;
            }
            out[(size_t)k * m->nowned + c] = v;
        }
    }
    return 0;
}
