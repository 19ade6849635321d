/*
 * rhs_general.cu - RHS of the coupled phase-field / chemistry / heat
 * equations on uniform grids: every problem the device accepts that the
 * phase-field-only kernels do not cover (chemical models, segregation
 * potentials, interface mobility factors, solute sources, heat conduction,
 * latent and specific heat, boundary faces, several interfaces).
 *
 * Replaces RHSFunction (src/cipher.c:27-681) with, in launch order
 * (launch_gen below):
 *   k_specialise, k_evaluate : the materials' T-series at the cells'
 *                 temperature (kept while it does not change);
 *   k_order_*   : the cells grouped by class (order.cuh);
 *   k_item_list, k_items (rhs_items.cu): the model evaluations of each
 *                 phase of the cells of several phases, one thread per
 *                 phase and part (energy; explicit potentials and tangent;
 *                 mobilities);
 *   k_chem_single / k_chem_cell (general_kernels.cuh): per cell
 *                 (src/cipher.c:148-233): site fractions of every active
 *                 phase at the cell's potentials, the interpolated
 *                 composition, lattice mobility (with the interface factors)
 *                 and conductivity, stored in scratch planes that the face
 *                 terms of both neighbours read;
 *   k_rhs_single (rhs_single.cu): the single-phase cells;
 *   k_rhs_general (general_kernels.cuh): the other cells: faces in the
 *                 reference's face order (phase, mu and heat fluxes,
 *                 235-317), boundary faces (319-389), then the cell terms
 *                 (391-664): capillary and chemical driving forces, active
 *                 set and constrained rate, dT/dt, dEX/dt and dmu/dt.
 * Every cell gives the same bits whichever kernel takes it.
 *
 * With an FP64 state (R = double) all arithmetic is FP64 in the reference's
 * operation order (this unit is compiled with --fmad=false).  With the mixed
 * layout (R = float: phi and T stored in FP32) the flux stencil (the
 * Andersson-Agren matrix times the potential difference, the heat-flux
 * product) and the interface terms (capillary force, active set, pair rates)
 * run in FP32, each face flux summed into an FP64 divergence, while the
 * model evaluations and the mu update stay FP64.  Gradient-based
 * anisotropy adds k_gradients before the RHS.  This unit also holds the
 * initial chemistry, nucleation and output-field kernels.
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "kernels.h"
#include "general_common.cuh"
#include "general_kernels.cuh"
#include "models.cuh"
#include "order.cuh"

namespace cipher {

/* ------------------------------------------------------------------ */
/* phase-field gradients (anisotropy)                                   */
/* ------------------------------------------------------------------ */

/* phase-field gradients of a cell's slots by least squares over its face
 * neighbours (src/cipher.c:82-146), with the weights the reference builds
 * once in main() (src/cipher.c:1232-1282) formed here per cell in the same
 * operation order: centroid differences in the cell's face order, AtA,
 * its closed-form inverse, (AtA)^-1 At.  grad[d][g] = sum_k w[d][k] (phi_k(g)
 * - phi(g)), the phase taken as absent (0) in a neighbour that does not
 * hold it; centroid differences across a periodic side are the raw ones, as
 * the reference's cell centroids give them. */
template <int PM, typename R>
__global__ void __launch_bounds__(kGenBlock) k_gradients(const GenArgs<R> a, const int DIM)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    const int64_t S = a.stride;
    int co[3] = {0, 0, 0};
    co[0] = (int)(c % a.res[0]);
    co[1] = DIM > 1 ? (int)((c / a.res[0]) % a.res[1]) : 0;
    co[2] = DIM > 2 ? (int)(c / ((int64_t)a.res[0] * a.res[1])) : 0;
    uint16_t ids[PM];
    double phi[PM];
    const int n = load_set<PM>(a, c, ids, phi);
    if (n == 0) return;
    /* neighbours in the cell's face order, with their centroid offsets */
    int64_t nbs[6];
    double A[6 * 3];
    int nls = 0;
    for (int f = 0; f < 3 * DIM; f++) {
        const int64_t nb = gen_face_nb(a.res, a.per, c, co, f, DIM);
        if (nb < 0 || nb == c) continue;
        const int64_t q[3] = {nb % a.res[0], DIM > 1 ? (nb / a.res[0]) % a.res[1] : 0,
                              DIM > 2 ? nb / ((int64_t)a.res[0] * a.res[1]) : 0};
        for (int d = 0; d < DIM; d++) {
            const double xn = ((double)q[d] + 0.5) * a.cw[d], xc = ((double)co[d] + 0.5) * a.cw[d];
            A[nls * DIM + d] = xn - xc;
        }
        nbs[nls++] = nb;
    }
    double ata[9], inv[9], w[3 * 6];
    for (int i = 0; i < DIM; i++)
        for (int j = i; j < DIM; j++) {
            double v = 0.0;
            for (int k = 0; k < nls; k++) v += A[k * DIM + i] * A[k * DIM + j];
            ata[i * DIM + j] = v;
            ata[j * DIM + i] = v;
        }
    invert_small(inv, ata, DIM);
    for (int i = 0; i < DIM; i++)
        for (int k = 0; k < nls; k++) {
            double v = 0.0;
            for (int d = 0; d < DIM; d++) v += inv[i * DIM + d] * A[k * DIM + d];
            w[i * nls + k] = v;
        }
    double gr[3][PM];
    for (int g = 0; g < n; g++)
        for (int d = 0; d < DIM; d++) {
            double t = 0.0;
            for (int k = 0; k < nls; k++) t -= w[d * nls + k] * phi[g];
            gr[d][g] = t;
        }
    for (int k = 0; k < nls; k++) {
        const int64_t nb = nbs[k];
        const int nn = a.as[nb];
        if (nn < 1 || nn > a.P) continue;          /* that cell's own thread raises the flag */
        int i = 0, j = 0;
        while (i < n && j < nn) {
            const uint16_t b = a.as[(int64_t)(1 + j) * S + nb];
            if (ids[i] == b) {
                const double pn = (double)a.phi[(int64_t)j * S + nb];
                for (int d = 0; d < DIM; d++) gr[d][i] += w[d * nls + k] * pn;
                i++;
                j++;
            } else if (ids[i] < b) {
                i++;
            } else {
                j++;
            }
        }
    }
    for (int d = 0; d < DIM; d++)
        for (int g = 0; g < n; g++) a.grad[((int64_t)d * a.P + g) * S + c] = gr[d][g];
}

/* ------------------------------------------------------------------ */
/* chemistry of the initial state                                       */
/* ------------------------------------------------------------------ */

template <int PM, typename R>
__global__ void __launch_bounds__(kGenBlock) k_chem_init(const GenArgs<R> a, double *ex, double *dp)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    const int64_t S = a.stride;
    uint16_t ids[PM];
    double phi[PM];
    const int n = load_set<PM>(a, c, ids, phi);
    if (n == 0) return;
    const double T = (double)a.tm[c];
    int own = 0;
    for (int g = 1; g < n; g++)
        if (phi[g] > phi[own]) own = g;
    for (int q = 0; q < a.P * a.SP; q++) ex[(int64_t)q * S + c] = 0.0;
    for (int g = 0; g < n; g++) {
        const cipher_material &mat = material_of(a.chem, ids[g]);
        double sp[2 * CIPHER_MAXCP];
        sitepot_explicit(a.chem, ids[g], mat.c0, T, sp);
        for (int q = 0; q < mat.nsites * a.ndp; q++) ex[(int64_t)(g * a.SP + q) * S + c] = sp[q];
    }
    const cipher_material &mo = material_of(a.chem, ids[own]);
    double sp[2 * CIPHER_MAXCP], mu[CIPHER_MAXCP];
    sitepot_total(a.chem, ids[own], mo.c0, T, sp);
    for (int d = 0; d < a.ndp; d++) mu[d] = 0.0;
    for (int s = 0; s < mo.nsites; s++)
        for (int d = 0; d < a.ndp; d++) mu[d] += sp[s * a.ndp + d];
    for (int d = 0; d < a.ndp; d++) dp[(int64_t)d * S + c] = mu[d];
}

/* ------------------------------------------------------------------ */
/* nucleation (src/cipher.c:715-867, src/material.c:150-290)            */
/* ------------------------------------------------------------------ */

/* one matrix phase of a nucleation cell (src/material.c:150-290): its site
 * fractions from the cell's implicit potentials stoichiometry*(mu - ci) - EX,
 * then h * chemical energy density (cnt) or h * the phase's average
 * composition (thermal), and h * R T M_raw into diff.  exslot points at the
 * slot's first EX plane at this cell (planes S apart). */
static __device__ __noinline__ void nuc_matrix_phase(const ChemTables ch, int phase, const double *exslot, int64_t S,
                                                     const double *mu, const double *ci, double T, double hg,
                                                     int cnt, double *matrixenergy, double *comp, double *diff)
{
    const cipher_material &mat = material_of(ch, phase);
    const int ncp = ch.ncp, ndp = ch.ndp;
    double pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP], mob[CIPHER_MAXCP];
    for (int s = 0; s < mat.nsites; s++)
        for (int d = 0; d < ndp; d++)
            pot[s * ndp + d] = mat.stoichiometry[s] * (mu[d] - ci[d]) - exslot[(int64_t)(s * ndp + d) * S];
    sitefrac(ch, phase, pot, T, y);
    if (cnt) {
        *matrixenergy += hg * energy_raw(mat, y, T, ncp) / mat.molarvolume;
    } else {
        for (int d = 0; d < ncp; d++) {
            double avg = 0.0;
            for (int s = 0; s < mat.nsites; s++) avg += mat.stoichiometry[s] * y[s * ncp + d];
            comp[d] += hg * avg;
        }
    }
    mobility_raw(mat, y, T, ncp, mob);
    for (int d = 0; d < ncp; d++) diff[d] += hg * CIPHER_R_GAS * T * mob[d];
}

/* chemical energy density of the nucleus phase at its c0 under the cell's
 * potentials (NucleationBarrier_cnt) */
static __device__ __noinline__ double nuc_phase_energy(const ChemTables ch, int phase, const double *mu,
                                                       const double *ci, double T)
{
    const cipher_material &ms = material_of(ch, phase);
    const int ndp = ch.ndp;
    double ex[2 * CIPHER_MAXCP], pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP];
    sitepot_explicit(ch, phase, ms.c0, T, ex);
    for (int s = 0; s < ms.nsites; s++)
        for (int d = 0; d < ndp; d++) pot[s * ndp + d] = ms.stoichiometry[s] * (mu[d] - ci[d]) - ex[s * ndp + d];
    sitefrac(ch, phase, pot, T, y);
    return energy_raw(ms, y, T, ch.ncp) / ms.molarvolume;
}

/* per listed cell of an active site: whether its phases are all matrix
 * phases of the site's nucleus, the nucleation barrier, the temperature and
 * the interpolated diffusivities of the nucleus model */
template <int PM, typename R>
__global__ void __launch_bounds__(kGenBlock) k_nuc_cells(const GenArgs<R> a, const NucArgs nu, int64_t nlist)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlist) return;
    const int site = nu.site_of[k];
    double *rec = nu.cellrec + k * (3 + a.ncp);
    for (int q = 0; q < 3 + a.ncp; q++) rec[q] = 0.0;
    if (!nu.active[site]) return;
    const int64_t c = nu.list[k], S = a.stride;
    uint16_t ids[PM];
    double phi[PM], h[PM];
    const int n = load_set<PM>(a, c, ids, phi);
    if (n == 0) return;
    const int model = nu.nuclei[nu.sitenucleus[site]].model;
    const int nmatrix = nu.nuclei[nu.sitenucleus[site]].nmatrix;
    const int32_t *matrix = nu.nuclei[nu.sitenucleus[site]].matrix;
    /* active phases within the matrix list (SetIntersection size == n) */
    int common = 0;
    for (int i = 0, j = 0; i < n && j < nmatrix;) {
        if (ids[i] == matrix[j]) { common++; i++; j++; }
        else if (ids[i] < matrix[j]) i++;
        else j++;
    }
    if (common != n) return;                      /* rec[0] = 0: the site retires */
    const double T = (double)a.tm[c];
    interpolant(a.interp, phi, n, h);
    double barrier = 0.0, diff[CIPHER_MAXCP];
    for (int d = 0; d < CIPHER_MAXCP; d++) diff[d] = 0.0;
    if (model == CIPHER_NUC_CNT || model == CIPHER_NUC_THERMAL) {
        const cipher_nucleus &nz = nu.nuclei[nu.sitenucleus[site]];
        double mu[CIPHER_MAXCP], ci[CIPHER_MAXCP], comp[CIPHER_MAXCP], matrixenergy = 0.0;
        for (int d = 0; d < CIPHER_MAXCP; d++) { mu[d] = 0.0; comp[d] = 0.0; }
        for (int d = 0; d < a.ndp; d++) mu[d] = a.dp[(int64_t)d * S + c];
        segregation(a, ids, h, n, ci);
        const int cnt = model == CIPHER_NUC_CNT;
        for (int g = 0; g < n; g++)
            nuc_matrix_phase(a.chem, ids[g], a.ex + (int64_t)g * a.SP * S + c, S, mu, ci, T, h[g], cnt,
                             &matrixenergy, comp, diff);
        if (cnt) {
            barrier = matrixenergy - nuc_phase_energy(a.chem, nu.sitephase[site], mu, ci, T);
        } else {
            double solvus = nz.solvus_temperature_0, enthalpy = nz.enthalpy_fusion_0;
            if (nz.has_solvus_c)
                for (int d = 0; d < a.ncp; d++) solvus += comp[d] * nz.solvus_temperature_c[d];
            if (nz.has_enthalpy_c)
                for (int d = 0; d < a.ncp; d++) enthalpy += comp[d] * nz.enthalpy_fusion_c[d];
            barrier = enthalpy * (1.0 - T / solvus);
        }
    }
    rec[0] = 1.0;
    rec[1] = barrier;
    rec[2] = T;
    for (int d = 0; d < a.ncp; d++) rec[3 + d] = diff[d];
}

/* one thread per site: the volume sums over its cells in list order */
__global__ void __launch_bounds__(128) k_nuc_sites(const NucArgs nu, int ncp)
{
    const int site = blockIdx.x * blockDim.x + threadIdx.x;
    if (site >= nu.nsites) return;
    double *out = nu.siterec + (int64_t)site * (4 + ncp);
    double ok = 1.0, vol = 0.0, tv = 0.0, gv = 0.0, dv[CIPHER_MAXCP];
    for (int d = 0; d < CIPHER_MAXCP; d++) dv[d] = 0.0;
    if (nu.active[site]) {
        for (int64_t k = nu.start[site]; k < nu.start[site + 1]; k++) {
            const double *rec = nu.cellrec + k * (3 + ncp);
            if (rec[0] == 0.0) { ok = 0.0; break; }
            vol += nu.vol;
            tv += nu.vol * rec[2];
            gv += nu.vol * rec[1];
            for (int d = 0; d < ncp; d++) dv[d] += nu.vol * rec[3 + d];
        }
    } else {
        ok = 0.0;
    }
    out[0] = ok;
    out[1] = vol;
    out[2] = tv;
    out[3] = gv;
    for (int d = 0; d < ncp; d++) out[4 + d] = dv[d];
}

/* cells of fired sites become their site's phase (src/cipher.c:831-851) */
template <typename R>
__global__ void __launch_bounds__(kGenBlock) k_nuc_reset(const GenArgs<R> a, const NucArgs nu, int64_t nlist)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlist) return;
    const int site = nu.site_of[k];
    if (!nu.fired[site]) return;
    const int64_t c = nu.list[k], S = a.stride;
    const int sp = nu.sitephase[site];
    uint16_t *as = (uint16_t *)a.as;
    as[c] = 1;
    as[S + c] = (uint16_t)sp;
    ((R *)a.phi)[c] = (R)1.0;
    if (a.ndp) {
        const double T = (double)a.tm[c];
        const cipher_material &ms = material_of(a.chem, sp);
        double ex[2 * CIPHER_MAXCP];
        sitepot_explicit(a.chem, sp, ms.c0, T, ex);
        for (int q = 0; q < ms.nsites * a.ndp; q++) ((double *)a.ex)[(int64_t)q * S + c] = ex[q];
    }
}

template <typename R>
static cudaError_t launch_nsums(const GenArgs<R> &a, const NucArgs &n, int64_t nlist, cudaStream_t s)
{
    if (nlist > 0) {
        k_nuc_cells<CIPHER_PMAX, R><<<(unsigned)((nlist + kGenBlock - 1) / kGenBlock), kGenBlock, 0, s>>>(a, n, nlist);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    k_nuc_sites<<<(n.nsites + 127) / 128, 128, 0, s>>>(n, a.ncp);
    return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_nreset(const GenArgs<R> &a, const NucArgs &n, int64_t nlist, cudaStream_t s)
{
    if (nlist < 1) return cudaSuccess;
    k_nuc_reset<R><<<(unsigned)((nlist + kGenBlock - 1) / kGenBlock), kGenBlock, 0, s>>>(a, n, nlist);
    return cudaGetLastError();
}

cudaError_t launch_nucleation_sums(const GenArgs<double> &a, const NucArgs &n, int64_t nlist, cudaStream_t s) { return launch_nsums(a, n, nlist, s); }
cudaError_t launch_nucleation_sums(const GenArgs<float> &a, const NucArgs &n, int64_t nlist, cudaStream_t s) { return launch_nsums(a, n, nlist, s); }
cudaError_t launch_nucleation_reset(const GenArgs<double> &a, const NucArgs &n, int64_t nlist, cudaStream_t s) { return launch_nreset(a, n, nlist, s); }
cudaError_t launch_nucleation_reset(const GenArgs<float> &a, const NucArgs &n, int64_t nlist, cudaStream_t s) { return launch_nreset(a, n, nlist, s); }

/* ------------------------------------------------------------------ */
/* output fields (src/cipher.c:976-1078)                                */
/* ------------------------------------------------------------------ */

template <int PM, typename R>
__global__ void __launch_bounds__(kGenBlock) k_output_fields(const GenArgs<R> a, const int32_t *kinds,
                                                             const int32_t *idx, int nf, double *out)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    const int64_t S = a.stride;
    uint16_t ids[PM];
    double phi[PM], h[PM];
    const int n = load_set<PM>(a, c, ids, phi);
    const double T = n > 0 ? (double)a.tm[c] : 0.0;
    if (n > 0) interpolant(a.interp, phi, n, h);
    double comp[CIPHER_MAXCP];
    bool have_comp = false;
    for (int k = 0; k < nf; k++) {
        double v = 0.0;
        const int kind = kinds[k], ix = idx[k];
        if (n == 0) {
            v = 0.0;
        } else if (kind == CIPHER_OUT_PHASEID || kind == CIPHER_OUT_MATID) {
            double mx = -CIPHER_LARGE;
            for (int g = 0; g < n; g++)
                if (h[g] > mx) {
                    mx = h[g];
                    v = kind == CIPHER_OUT_PHASEID ? (double)ids[g] : (double)a.chem.pmm[ids[g]];
                }
        } else if (kind == CIPHER_OUT_INTERFACEID) {
            v = -1.0;
            for (int k2 = 0; k2 < n; k2++)
                for (int j = k2 + 1; j < n; j++) v = (double)a.itflist[ids[k2] * a.npf + ids[j]];
        } else if (kind == CIPHER_OUT_CHEMPOT) {
            v = (ix >= 0 && ix < a.ndp) ? a.dp[(int64_t)ix * S + c] : 0.0;
        } else if (kind == CIPHER_OUT_COMP) {
            if (!have_comp) {
                for (int d = 0; d < CIPHER_MAXCP; d++) comp[d] = 0.0;
                if (a.ndp) {
                    double mu[CIPHER_MAXCP], ci[CIPHER_MAXCP];
                    for (int d = 0; d < a.ndp; d++) mu[d] = a.dp[(int64_t)d * S + c];
                    segregation(a, ids, h, n, ci);
                    for (int g = 0; g < n; g++) {
                        const cipher_material &mat = material_of(a.chem, ids[g]);
                        double pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP];
                        slot_potential(a, mat, mu, ci, c, g, pot);
                        sitefrac(a.chem, ids[g], pot, T, y);
                        for (int s2 = 0; s2 < mat.nsites; s2++)
                            for (int d = 0; d < a.ncp; d++)
                                comp[d] += h[g] * mat.stoichiometry[s2] * y[s2 * a.ncp + d];
                    }
                }
                have_comp = true;
            }
            v = (ix >= 0 && ix < a.ncp) ? comp[ix] : 0.0;
        } else if (kind == CIPHER_OUT_PHI) {
            for (int g = 0; g < n; g++)
                if ((int)ids[g] == ix) v = phi[g];
        } else if (kind == CIPHER_OUT_TEMPERATURE) {
            v = T;
        }
        out[(int64_t)k * a.ncells + c] = v;
    }
}

template <typename R>
static cudaError_t launch_out(const GenArgs<R> &a, const int32_t *kinds, const int32_t *idx, int nf, double *out,
                              cudaStream_t s)
{
    const unsigned blocks = (unsigned)((a.ncells + kGenBlock - 1) / kGenBlock);
    k_output_fields<CIPHER_PMAX, R><<<blocks, kGenBlock, 0, s>>>(a, kinds, idx, nf, out);
    return cudaGetLastError();
}

cudaError_t launch_output_fields(const GenArgs<double> &a, const int32_t *kinds, const int32_t *idx, int nf,
                                 double *out, cudaStream_t s) { return launch_out(a, kinds, idx, nf, out, s); }
cudaError_t launch_output_fields(const GenArgs<float> &a, const int32_t *kinds, const int32_t *idx, int nf,
                                 double *out, cudaStream_t s) { return launch_out(a, kinds, idx, nf, out, s); }

/* ------------------------------------------------------------------ */
/* materials specialised at one temperature                             */
/* ------------------------------------------------------------------ */

/* T-series slot k of a material (0 <= k < kSpecSlots), or NULL.  Quadratic
 * materials keep their unary and quadratic series, whose T-derivatives the
 * tangent needs. */
constexpr int kSpecSlots = 1 + CIPHER_MAXCP * CIPHER_MAXCP + 4 * CIPHER_MAXRKTAB * CIPHER_MAXRK +
                           CIPHER_MAXCP * (CIPHER_MAXCP + CIPHER_MAXBIN * CIPHER_MAXRK) + 3;

__device__ inline cipher_tseries *spec_slot(cipher_material &m, int k)
{
    if (k == 0) return &m.ref;
    k -= 1;
    if (k < CIPHER_MAXCP * CIPHER_MAXCP) return m.model == CIPHER_CHEM_QUADRATIC ? nullptr : &m.unary[k];
    k -= CIPHER_MAXCP * CIPHER_MAXCP;
    if (k < 4 * CIPHER_MAXRKTAB * CIPHER_MAXRK) {
        const int tab = k / (CIPHER_MAXRKTAB * CIPHER_MAXRK), e = k % (CIPHER_MAXRKTAB * CIPHER_MAXRK);
        cipher_rk *rk = tab == 0 ? m.binary : tab == 1 ? m.ternary : tab == 2 ? m.binaryq : m.ternaryq;
        return &rk[e / CIPHER_MAXRK].h[e % CIPHER_MAXRK];
    }
    k -= 4 * CIPHER_MAXRKTAB * CIPHER_MAXRK;
    if (k < CIPHER_MAXCP * (CIPHER_MAXCP + CIPHER_MAXBIN * CIPHER_MAXRK)) {
        cipher_mobility &mob = m.mobilityc[k / (CIPHER_MAXCP + CIPHER_MAXBIN * CIPHER_MAXRK)];
        const int e = k % (CIPHER_MAXCP + CIPHER_MAXBIN * CIPHER_MAXRK);
        if (e < CIPHER_MAXCP) return &mob.unary[e];
        const int b = e - CIPHER_MAXCP;
        return &mob.binary[b / CIPHER_MAXRK].h[b % CIPHER_MAXRK];
    }
    k -= CIPHER_MAXCP * (CIPHER_MAXCP + CIPHER_MAXBIN * CIPHER_MAXRK);
    if (k == 0) return &m.specific_heat;
    if (k == 1) return &m.latent_heat;
    if (k == 2) return &m.tconductivity;
    return nullptr;
}

/* one block per material: copy it, then replace each T-series s by the
 * constant series {n = 1, T^0: tseries(T, s)} at T = the first cell's
 * temperature.  A constant series evaluates to 0.0 + v = v, so every model
 * function returns the same bits from either copy; cells at another
 * temperature keep reading the original.  tspec[0]: the temperature of the
 * copies; tspec[1 + m]: of material m's copy, which is kept when T has not
 * changed (the materials are fixed for the context's life). */
template <typename R>
__global__ void __launch_bounds__(256) k_specialise(const cipher_material *mat, cipher_material *spec, const R *tm,
                                                    double *tspec)
{
    const double T = (double)tm[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) tspec[0] = T;
    if (tspec[1 + blockIdx.x] == T) return;
    const double *src = (const double *)&mat[blockIdx.x];
    double *dst = (double *)&spec[blockIdx.x];
    for (size_t i = threadIdx.x; i < sizeof(cipher_material) / sizeof(double); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    cipher_material &m = spec[blockIdx.x];
    const cipher_material &o = mat[blockIdx.x];
    for (int k = threadIdx.x; k < kSpecSlots; k += blockDim.x) {
        cipher_tseries *ts = spec_slot(m, k);
        if (!ts) continue;
        /* the matching slot of the original: same offset */
        const cipher_tseries *os = (const cipher_tseries *)((const char *)&o + ((const char *)ts - (const char *)&m));
        if (os->n == 0 && os->logcoeff == 0.0) continue;
        const double v = tseries(T, *os);
        ts->n = 1;
        ts->exp[0] = 0;
        ts->coeff[0] = v;
        ts->logcoeff = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) tspec[1 + blockIdx.x] = T;
}

/* one block per material: the evaluated tables (MatV) of the specialised
 * copy, each value tseries(T, s) of the specialised series s at the
 * specialisation temperature - the value the model bodies compute from
 * that series, bit for bit.  tspec[1 + nmat + m]: the temperature of
 * material m's tables, kept while it has not changed. */
__global__ void __launch_bounds__(256) k_evaluate(const cipher_material *spec, MatV *mv, double *tspec)
{
    const double T = tspec[0];
    double *done = &tspec[1 + gridDim.x + blockIdx.x];
    if (*done == T) return;
    const cipher_material &m = spec[blockIdx.x];
    MatV &v = mv[blockIdx.x];
    const int t = threadIdx.x, nt = blockDim.x;
    if (t == 0) {
        v.model = m.model;
        v.p = m.p;
        v.q = m.q;
        v.molarvolume = m.molarvolume;
        v.stoichiometry[0] = m.stoichiometry[0];
        v.stoichiometry[1] = m.stoichiometry[1];
        v.ref.v = tseries(T, m.ref);
    }
    for (int k = t; k < CIPHER_MAXCP * CIPHER_MAXCP; k += nt) v.unary[k].v = tseries(T, m.unary[k]);
    for (int k = t; k < CIPHER_MAXCP; k += nt) {
        v.quad_ceq[k].v = 0.0;
        v.quad_binary[k].v = 0.0;
    }
    auto rk = [&](RkV &o, const cipher_rk &r) {
        o.n = r.n;
        for (int j = 0; j < CIPHER_MAXRK; j++) {
            o.i[j] = r.i[j];
            o.h[j].v = tseries(T, r.h[j]);
        }
    };
    for (int k = t; k < 4 * CIPHER_MAXRKTAB; k += nt) {
        const int tab = k / CIPHER_MAXRKTAB, e = k % CIPHER_MAXRKTAB;
        if (tab == 0) rk(v.binary[e], m.binary[e]);
        else if (tab == 1) rk(v.ternary[e], m.ternary[e]);
        else if (tab == 2) rk(v.binaryq[e], m.binaryq[e]);
        else rk(v.ternaryq[e], m.ternaryq[e]);
    }
    for (int k = t; k < CIPHER_MAXCP * (1 + CIPHER_MAXBIN); k += nt) {
        const int c = k / (1 + CIPHER_MAXBIN), e = k % (1 + CIPHER_MAXBIN);
        const cipher_mobility &mo = m.mobilityc[c];
        MobV &vo = v.mobilityc[c];
        if (e == 0) {
            vo.m0 = mo.m0;
            for (int j = 0; j < CIPHER_MAXCP; j++) vo.unary[j].v = tseries(T, mo.unary[j]);
        } else {
            rk(vo.binary[e - 1], mo.binary[e - 1]);
        }
    }
    __syncthreads();
    if (t == 0) *done = T;
}

/* ------------------------------------------------------------------ */
/* launchers                                                            */
/* ------------------------------------------------------------------ */

template <typename R>
static cudaError_t launch_gen(const GenArgs<R> &a, int dim, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((a.ncells + kGenBlock - 1) / kGenBlock);
    const unsigned wblocks = (unsigned)((a.ncells + kWarpBlock - 1) / kWarpBlock);
    if (a.chem.spec) {
        k_specialise<R><<<a.chem.nmat, 256, 0, s>>>(a.chem.mat, (cipher_material *)a.chem.spec, a.tm,
                                                     (double *)a.chem.tspec);
        if (a.chem.matv_tab)
            k_evaluate<<<a.chem.nmat, 256, 0, s>>>(a.chem.spec, (MatV *)a.chem.matv_tab, (double *)a.chem.tspec);
    }
    if (a.order) {
        const OrderBuf o = {a.order, a.order_counts, a.order_cursor, a.nclass, a.ncells};
        launch_order(o, GeneralClassKey{a.as, a.stride, a.chem.pmm, a.npf, a.chem.nmat}, s);
    }
    /* the phase items of the cells of several phases (they read only the
     * state); composition, mobility and conductivity of every cell before
     * any face flux reads them (k_chem_cell combines the items' mobilities);
     * then the RHS of the single-phase cells and of the rest */
    cudaError_t e;
    if (a.icap && (e = launch_items(a, s)) != cudaSuccess) return e;
    if (a.ndp) {
        if (a.single_models && (e = launch_chem_single(a, s)) != cudaSuccess) return e;
        k_chem_cell<CIPHER_PMAX, R><<<wblocks, kWarpBlock, 0, s>>>(a);
    }
    if (a.grad) k_gradients<CIPHER_PMAX, R><<<blocks, kGenBlock, 0, s>>>(a, dim);
    if (a.single_models && (e = launch_rhs_single(a, dim, s)) != cudaSuccess) return e;
    k_rhs_general<CIPHER_PMAX, R><<<wblocks, 2 * kWarpBlock, 0, s>>>(a, dim);   /* a face and a cell warp */
    return cudaGetLastError();
}

cudaError_t launch_rhs_general(const GenArgs<double> &a, int dim, cudaStream_t s) { return launch_gen(a, dim, s); }
cudaError_t launch_rhs_general(const GenArgs<float> &a, int dim, cudaStream_t s) { return launch_gen(a, dim, s); }

template <typename R>
static cudaError_t launch_init(const GenArgs<R> &a, double *ex, double *dp, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((a.ncells + kGenBlock - 1) / kGenBlock);
    k_chem_init<CIPHER_PMAX, R><<<blocks, kGenBlock, 0, s>>>(a, ex, dp);
    return cudaGetLastError();
}

cudaError_t launch_chem_init(const GenArgs<double> &a, double *ex, double *dp, cudaStream_t s) { return launch_init(a, ex, dp, s); }
cudaError_t launch_chem_init(const GenArgs<float> &a, double *ex, double *dp, cudaStream_t s) { return launch_init(a, ex, dp, s); }

}  // namespace cipher
