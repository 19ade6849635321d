/*
 * rhs_general.cu - RHS of the coupled phase-field / chemistry / heat
 * equations on uniform grids: every problem the device accepts that the
 * phase-field-only kernels do not cover (chemical models, segregation
 * potentials, interface mobility factors, solute sources, heat conduction,
 * latent and specific heat, boundary faces, several interfaces).
 *
 * Replaces RHSFunction (src/cipher.c:27-681) in two launches:
 *   k_chem_cell : per cell (src/cipher.c:148-233): site fractions of every
 *                 active phase at the cell's potentials, the interpolated
 *                 composition, lattice mobility (with the interface factors)
 *                 and conductivity, stored in scratch planes that the face
 *                 terms of both neighbours read;
 *   k_rhs_general: per cell: the cell's faces gathered in the reference's
 *                 face order (phase, mu and heat fluxes, 235-317), its
 *                 boundary faces (319-389), then the cell terms (391-664):
 *                 capillary and chemical driving forces, active set and
 *                 constrained rate, dT/dt, dEX/dt and dmu/dt.
 * Site fractions of the cell's own phases are recomputed in the second
 * kernel instead of stored: the same arithmetic gives the same bits, and a
 * few exponentials per phase cost less than 8*P*S bytes written and read.
 *
 * With an FP64 state (R = double) all arithmetic is FP64 in the reference's
 * operation order (this unit is compiled with --fmad=false).  With the mixed
 * layout (R = float: phi and T stored in FP32) the flux stencil (the
 * Andersson-Agren matrix times the potential difference, the heat-flux
 * product) and the interface terms (capillary force, active set, pair rates)
 * run in FP32, each face flux summed into an FP64 divergence, while the
 * model evaluations and the mu update stay FP64.  Gradient-based
 * anisotropy adds k_gradients before the RHS; both kernels walk the cells
 * grouped by class (k_order_*).
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "kernels.h"
#include "models.cuh"
#include "order.cuh"

namespace cipher {

constexpr int kGenBlock = 128;

/* phase interpolant h and its transposed derivative (src/utility.c:470-557) */
__device__ inline void interpolant(int kind, const double *phi, int n, double *h)
{
    if (kind == CIPHER_INTERP_LINEAR) {
        for (int g = 0; g < n; g++) h[g] = phi[g];
        return;
    }
    if (n == 1) { h[0] = 1.0; return; }
    double sum = 0.0;
    for (int g = 0; g < n; g++) {
        h[g] = kind == CIPHER_INTERP_QUADRATIC ? phi[g] * phi[g] : phi[g] * phi[g] * (3.0 - 2.0 * phi[g]);
        sum += h[g];
    }
    for (int g = 0; g < n; g++) h[g] /= sum;
}

template <int PM>
__device__ inline void interpolant_dT(int kind, double *v, const double *phi, int n)
{
    if (kind == CIPHER_INTERP_LINEAR) return;
    if (n == 1) { v[0] = 0.0; return; }
    double avg = 0.0, sum = 0.0;
    for (int g = 0; g < n; g++) {
        double w = kind == CIPHER_INTERP_QUADRATIC ? phi[g] * phi[g] : phi[g] * phi[g] * (3.0 - 2.0 * phi[g]);
        sum += w;
        avg += w * v[g];
    }
    for (int g = 0; g < n; g++) {
        if (kind == CIPHER_INTERP_QUADRATIC) v[g] = 2.0 * phi[g] * (v[g] - avg / sum) / sum;
        else v[g] = 6.0 * phi[g] * (1.0 - phi[g]) * (v[g] - avg / sum) / sum;
    }
}

template <typename R>
__device__ __forceinline__ const DevInterface &pair_itf(const GenArgs<R> &a, int ia, int ib)
{
    return a.itfs[a.itflist[ia * a.npf + ib]];
}

/* implicit site potentials of slot g: stoichiometry*(mu - ci) - EX */
template <typename R>
__device__ __forceinline__ void slot_potential(const GenArgs<R> &a, const cipher_material &mat, const double *mu,
                                               const double *ci, int64_t c, int g, double *pot)
{
    const int64_t S = a.stride;
    for (int s = 0; s < mat.nsites; s++)
        for (int d = 0; d < a.ndp; d++)
            pot[s * a.ndp + d] = mat.stoichiometry[s] * (mu[d] - ci[d]) -
                                 a.ex[(int64_t)(g * a.SP + s * a.ndp + d) * S + c];
}

/* segregation potential of the cell, sum_{k<j} h_k h_j V_kj (src/cipher.c:160-172) */
template <typename R>
__device__ __forceinline__ void segregation(const GenArgs<R> &a, const uint16_t *ids, const double *h, int n,
                                            double *ci)
{
    for (int d = 0; d < CIPHER_MAXCP; d++) ci[d] = 0.0;
    for (int k = 0; k < n; k++)
        for (int j = k + 1; j < n; j++) {
            const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
            if (itf.has_potential)
                for (int d = 0; d < a.ndp; d++) ci[d] += h[k] * h[j] * itf.potential[d];
        }
}

/* read a cell's set; returns n, or 0 (and raises ERR_BADSET) if invalid */
template <int PM, typename R>
__device__ __forceinline__ int load_set(const GenArgs<R> &a, int64_t c, uint16_t *ids, double *phi)
{
    const int64_t S = a.stride;
    int n = a.as[c];
    if (n < 1 || n > a.P || n > PM) {
        atomicOr(a.err, ERR_BADSET);
        return 0;
    }
    for (int g = 0; g < n; g++) {
        ids[g] = a.as[(int64_t)(1 + g) * S + c];
        phi[g] = (double)a.phi[(int64_t)g * S + c];
        if (ids[g] >= a.npf) {
            atomicOr(a.err, ERR_BADSET);
            return 0;
        }
    }
    return n;
}

/* ------------------------------------------------------------------ */
/* per-cell composition, mobility and conductivity                      */
/* ------------------------------------------------------------------ */

template <int PM, typename R>
__global__ void __launch_bounds__(kGenBlock) k_chem_cell(const GenArgs<R> a)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ncells) return;
    const int64_t c = a.order ? (int64_t)a.order[t] : t;
    const int64_t S = a.stride;
    const int ncp = a.ncp, ndp = a.ndp;
    uint16_t ids[PM];
    double phi[PM], h[PM];
    const int n = load_set<PM>(a, c, ids, phi);
    double mu[CIPHER_MAXCP], ci[CIPHER_MAXCP], mm[CIPHER_MAXCP], cc[CIPHER_MAXCP];
    for (int d = 0; d < CIPHER_MAXCP; d++) { mm[d] = 0.0; cc[d] = 0.0; }
    double tc = 0.0;
    if (n > 0) {
        const double T = (double)a.tm[c];
        const ChemTables ch = chem_at(a.chem, T);
        for (int d = 0; d < ndp; d++) mu[d] = a.dp[(int64_t)d * S + c];
        interpolant(a.interp, phi, n, h);
        segregation(a, ids, h, n, ci);
        for (int g = 0; g < n; g++) {
            const cipher_material &mat = material_of(ch, ids[g]);
            double pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP], me[CIPHER_MAXCP];
            slot_potential(a, mat, mu, ci, c, g, pot);
            sitefrac(ch, ids[g], pot, T, y);
            mobility(ch, ids[g], y, T, me);
            for (int d = 0; d < ncp; d++) mm[d] += h[g] * me[d];
            for (int s = 0; s < mat.nsites; s++)
                for (int d = 0; d < ncp; d++) cc[d] += h[g] * mat.stoichiometry[s] * y[s * ncp + d];
            if (mat.tconductivity.n) tc += h[g] * tseries(T, mat.tconductivity);
        }
        for (int k = 0; k < n; k++)
            for (int j = k + 1; j < n; j++) {
                const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
                if (itf.has_mobilityc)
                    for (int d = 0; d < ncp; d++) mm[d] *= exp(itf.mobilityc[d] / CIPHER_R_GAS / T);
            }
    }
    for (int d = 0; d < ncp; d++) {
        a.comp[(int64_t)d * S + c] = cc[d];
        a.mob[(int64_t)d * S + c] = mm[d];
    }
    a.tcond[c] = tc;
}

/* ------------------------------------------------------------------ */
/* cell grouping: the general kernels process cells grouped by class    */
/* ------------------------------------------------------------------ */

/* A warp of the general kernels runs one model per lane: cells whose single
 * phase belongs to different materials, and cells with several phases,
 * diverge.  The kernels therefore walk the cells grouped by class (the
 * material of a single-phase cell; sets of 2, 3, more phases; order.cuh).
 * Every cell's arithmetic is unchanged: the results do not depend on the
 * order. */
struct GeneralClassKey {
    const uint16_t *as;
    int64_t stride;
    const int32_t *pmm;
    int npf, nmat;
    __device__ __forceinline__ int operator()(int64_t c) const
    {
        const int n = as[c];
        if (n == 1) {
            const int id = as[stride + c];
            if (id >= 0 && id < npf) {
                const int m = pmm[id];
                if (m >= 0 && m < nmat) return m;
            }
        }
        return nmat + (n <= 2 ? 0 : n == 3 ? 1 : 2);
    }
};

/* ------------------------------------------------------------------ */
/* the RHS                                                              */
/* ------------------------------------------------------------------ */

/* neighbour at face position f in the reference's face order: [0,DIM)
 * below without wrap (descending d), [DIM,2DIM) own faces (ascending d),
 * [2DIM,3DIM) wrapped around from above (ascending d); -1 if absent */
__device__ __forceinline__ int64_t gen_face_nb(const int *res, const int *per, int64_t c, const int *co, int f,
                                               const int DIM)
{
    const int64_t st[3] = {1, (int64_t)res[0], (int64_t)res[0] * res[1]};
    if (f < DIM) {
        const int e = DIM - 1 - f;
        return co[e] > 0 ? c - st[e] : -1;
    }
    if (f < 2 * DIM) {
        const int d = f - DIM;
        if (co[d] < res[d] - 1) return c + st[d];
        return (per[d] && res[d] > 1) ? c - (int64_t)(res[d] - 1) * st[d] : -1;
    }
    const int d = f - 2 * DIM;
    return (co[d] == 0 && per[d] && res[d] > 1) ? c + (int64_t)(res[d] - 1) * st[d] : -1;
}

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

/* ff*x/vol as the reference forms it (src/cipher.c:281-282) */
template <typename R>
__device__ __forceinline__ double face_div(const GenArgs<R> &a, double x)
{
    if (a.geom_mode == 2) return x;
    if (a.geom_mode == 1) return (a.ffactor * x) * a.inv_vol;
    return (a.ffactor * x) / a.vol;
}

template <int PM, typename R>
__global__ void __launch_bounds__(kGenBlock, 12) k_rhs_general(const GenArgs<R> a, const int DIM)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ncells) return;
    const int64_t c = a.order ? (int64_t)a.order[t] : t;
    const int64_t S = a.stride;
    const int ncp = a.ncp, ndp = a.ndp, SP = a.SP;
    const double PI = CIPHER_PI_D;
    const bool listed = a.fl.start != nullptr;   /* an adapted mesh: faces from the lists */
    int co[3] = {0, 0, 0};
    if (!listed) {
        co[0] = (int)(c % a.res[0]);
        co[1] = DIM > 1 ? (int)((c / a.res[0]) % a.res[1]) : 0;
        co[2] = DIM > 2 ? (int)(c / ((int64_t)a.res[0] * a.res[1])) : 0;
    }

    uint16_t ids[PM];
    double phi[PM], h[PM], lap[PM], pf[PM];
    const int n = load_set<PM>(a, c, ids, phi);
    if (n == 0) return;
    const double T = (double)a.tm[c];
    const ChemTables ch = chem_at(a.chem, T);
    double mu[CIPHER_MAXCP], ldp[CIPHER_MAXCP];
    for (int d = 0; d < ndp; d++) { mu[d] = a.dp[(int64_t)d * S + c]; ldp[d] = 0.0; }
    double ltm = 0.0;
    for (int g = 0; g < n; g++) lap[g] = 0.0;

    /* ---- faces in the reference's face order (src/cipher.c:235-317) ---- */
    const int f0 = listed ? a.fl.start[c] : 0, f1 = listed ? a.fl.start[c + 1] : 3 * DIM;
    const double vol_c = listed ? a.fl.vol[c] : 0.0;
#pragma unroll 1
    for (int f = f0; f < f1; f++) {
        int64_t nb;
        bool self_L;
        double ffv = 0.0;
        if (listed) {
            const int32_t v = a.fl.nbr[f];
            nb = v & 0x7fffffff;
            self_L = (v & FACE_SELF_L) != 0;
            ffv = a.fl.ff[a.fl.face[f]];
        } else {
            nb = gen_face_nb(a.res, a.per, c, co, f, DIM);
            if (nb < 0) continue;
            self_L = f >= DIM && f < 2 * DIM;
        }
        /* ff*x/vol of this cell, as the reference forms it (src/cipher.c:281-282) */
        auto fdiv = [&](double x) { return listed ? (ffv * x) / vol_c : face_div(a, x); };
        const int64_t cl = self_L ? c : nb, cr = self_L ? nb : c;
        const int nn = a.as[nb];
        if (nn < 1 || nn > a.P) continue;          /* that cell's own thread raises the flag */
        /* phase flux, gated on the L cell only (src/cipher.c:277) */
        const bool gate = self_L ? (n > 1 || ids[0] > 1) : (nn > 1 || a.as[S + nb] > 1);
        if (gate) {
            int i = 0, j = 0;
            while (i < n && j < nn) {
                const uint16_t b = a.as[(int64_t)(1 + j) * S + nb];
                if (ids[i] == b) {
                    const double pn = (double)a.phi[(int64_t)j * S + nb];
                    if (self_L) lap[i] += fdiv(pn - phi[i]);
                    else lap[i] -= fdiv(phi[i] - pn);
                    i++;
                    j++;
                } else if (ids[i] < b) {
                    i++;
                } else {
                    j++;
                }
            }
        }
        /* chemical-potential flux with the Andersson-Agren frame (material.c:1125-1137) */
        if (ndp) {
            double me[CIPHER_MAXCP], ca[CIPHER_MAXCP];
            for (int d = 0; d < ncp; d++) {
                const double ml = a.mob[(int64_t)d * S + cl], mr = a.mob[(int64_t)d * S + cr];
                const double cL = a.comp[(int64_t)d * S + cl], cR = a.comp[(int64_t)d * S + cr];
                if (fabs(ml) > 1e-32 && fabs(mr) > 1e-32) me[d] = 2.0 * ml * mr / (ml + mr);
                else me[d] = 0.0;
                ca[d] = 2.0 * cL * cR / (cL + cR);
            }
            if constexpr (sizeof(R) == 4) {
                /* mixed: the flux stencil in FP32 - the Andersson-Agren matrix
                 * and its product with the potential difference (formed in
                 * FP64, then rounded) - accumulated into the FP64 divergence */
                float MB[(CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1)], dmu[CIPHER_MAXCP];
                for (int i = 0; i < ndp; i++)
                    for (int j = 0; j < ndp; j++) {
                        float acc = 0.0f;
                        for (int k = 0; k < ncp; k++)
                            acc += ((j == k ? 1.0f : 0.0f) - (float)ca[j]) * ((k == i ? 1.0f : 0.0f) - (float)ca[i]) *
                                   (float)me[k];
                        MB[i * ndp + j] = acc;
                    }
                for (int d = 0; d < ndp; d++) dmu[d] = (float)(a.dp[(int64_t)d * S + cr] - a.dp[(int64_t)d * S + cl]);
                for (int d = 0; d < ndp; d++) {
                    float f = 0.0f;
                    for (int j = 0; j < ndp; j++) f += MB[d * ndp + j] * dmu[j];
                    if (self_L) ldp[d] += fdiv((double)f);
                    else ldp[d] -= fdiv((double)f);
                }
            } else {
                double MB[(CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1)], dmu[CIPHER_MAXCP], fl[CIPHER_MAXCP];
                for (int i = 0; i < ndp; i++)
                    for (int j = 0; j < ndp; j++) {
                        double acc = 0.0;
                        for (int k = 0; k < ncp; k++)
                            acc += ((j == k ? 1.0 : 0.0) - ca[j]) * ((k == i ? 1.0 : 0.0) - ca[i]) * me[k];
                        MB[i * ndp + j] = acc;
                    }
                for (int d = 0; d < ndp; d++) dmu[d] = a.dp[(int64_t)d * S + cr] - a.dp[(int64_t)d * S + cl];
                matvec(fl, MB, dmu, ndp);
                for (int d = 0; d < ndp; d++) {
                    if (self_L) ldp[d] += fdiv(fl[d]);
                    else ldp[d] -= fdiv(fl[d]);
                }
            }
        }
        /* heat flux (mixed: the face product in FP32) */
        if (a.tcond) {
            const double tl = a.tcond[cl], tr = a.tcond[cr];
            if (fabs(tl) > 1e-32 && fabs(tr) > 1e-32) {
                double ft;
                if constexpr (sizeof(R) == 4)
                    ft = (double)((float)(2.0 * tl * tr / (tl + tr)) * ((float)a.tm[cr] - (float)a.tm[cl]));
                else
                    ft = 2.0 * tl * tr / (tl + tr) * ((double)a.tm[cr] - (double)a.tm[cl]);
                if (self_L) ltm += fdiv(ft);
                else ltm -= fdiv(ft);
            }
        }
    }

    /* ---- boundary faces (src/cipher.c:319-389) ---- */
    if (a.nbcs) {
        const double dc = listed ? a.fl.delta[c] : a.delta;
        const double cf = 1.0 / ipow(dc, 2);
        const double tcc = a.tcond ? a.tcond[c] : 0.0;
        const int q0 = listed ? a.fl.bstart[c] : 0, q1 = listed ? a.fl.bstart[c + 1] : 2 * DIM;
        for (int b = 0; b < a.nbcs; b++) {
            const DevBC &bc = a.bcs[b];
#pragma unroll 1
            for (int q = q0; q < q1; q++) {
                if (listed) {
                    if (bc.label != a.fl.blabel[q]) continue;
                } else {
                    const int d = q >> 1;
                    if (a.per[d]) continue;
                    const bool on = (q & 1) ? co[d] == a.res[d] - 1 : co[d] == 0;
                    if (!on || bc.label != 2 * d + 1 + (q & 1)) continue;
                }
                double fd[CIPHER_MAXCP];
                for (int k = 0; k < CIPHER_MAXCP; k++) fd[k] = 0.0;
                if (bc.chem_type != CIPHER_BC_NONE) {
                    if (bc.chem_type == CIPHER_BC_NEUMANN) {
                        for (int k = 0; k < ndp; k++) if (bc.chem_on[k]) fd[k] = bc.chem_val[k] * dc;
                    } else {
                        for (int k = 0; k < ndp; k++)
                            if (bc.chem_on[k]) fd[k] = a.mob[(int64_t)k * S + c] * (bc.chem_val[k] - mu[k]);
                    }
                }
                double fluxt = 0.0;
                if (bc.thermal_type == CIPHER_BC_NEUMANN) fluxt = tcc * bc.thermal_val * dc;
                else if (bc.thermal_type == CIPHER_BC_DIRICHLET) fluxt = tcc * (bc.thermal_val - T);
                if (bc.chem_type != CIPHER_BC_NONE)
                    for (int k = 0; k < ndp; k++) ldp[k] += cf * fd[k];
                if (bc.thermal_type != CIPHER_BC_NONE) ltm += cf * fluxt;
            }
        }
    }

    /* ---- cell terms (src/cipher.c:391-664) ---- */
    interpolant(a.interp, phi, n, h);
    double ci[CIPHER_MAXCP];
    if (ndp) segregation(a, ids, h, n, ci);

    /* pass over the phases: driving force, dEX/dt and the tangent sum */
    double chem[PM], yw[PM * (CIPHER_MAXCP - 1)];
    double cbar[CIPHER_MAXCP], dcdm[(CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1)];
    for (int d = 0; d < CIPHER_MAXCP; d++) cbar[d] = 0.0;
    for (int q = 0; q < (CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1); q++) dcdm[q] = 0.0;
    /* tangent of the last phase evaluated: reused by the composition rate
     * below when the cell has a single phase (same arguments, same bits) */
    double tpot[2 * 16], tex[2 * 16], tT[2 * CIPHER_MAXCP];
    for (int g = 0; g < n; g++) {
        const cipher_material &mat = material_of(ch, ids[g]);
        double pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP];
        if (ndp) {
            slot_potential(a, mat, mu, ci, c, g, pot);
            sitefrac(ch, ids[g], pot, T, y);
        }
        if (n > 1) {
            chem[g] = chemenergy(ch, ids[g], y, mu, T);
            for (int s = 0; s < mat.nsites; s++)
                for (int d = 0; d < ndp; d++) cbar[d] += h[g] * mat.stoichiometry[s] * y[s * ncp + d];
        }
        if (ndp) {
            for (int d = 0; d < ndp; d++) {
                double w = 0.0;
                for (int s = 0; s < mat.nsites; s++) w += mat.stoichiometry[s] * y[s * ncp + d];
                yw[g * (CIPHER_MAXCP - 1) + d] = w;
            }
            /* explicit potential relaxation (src/cipher.c:570-581) */
            double spx[2 * CIPHER_MAXCP];
            sitepot_explicit(ch, ids[g], y, T, spx);
            for (int s = 0; s < mat.nsites; s++)
                for (int d = 0; d < ndp; d++) {
                    const int64_t pl = (int64_t)(g * SP + s * ndp + d) * S + c;
                    a.fex[pl] = mat.chempot_ex_kineticcoeff * (spx[s * ndp + d] - a.ex[pl]);
                }
            for (int q = mat.nsites * ndp; q < SP; q++) a.fex[(int64_t)(g * SP + q) * S + c] = 0.0;
            sitefrac_tangent(ch, ids[g], y, pot, T, tpot, tex, tT);
            for (int s = 0; s < mat.nsites; s++)
                for (int q = 0; q < ndp * ndp; q++)
                    dcdm[q] += h[g] * mat.stoichiometry[s] * mat.stoichiometry[s] * tpot[s * ndp * ndp + q];
        }
    }
    for (int q = n * SP; q < a.P * SP; q++) a.fex[(int64_t)q * S + c] = 0.0;

    /* pair properties; with anisotropy they depend on the pair's normal,
     * the normalised difference of the two slots' gradients (src/cipher.c:
     * 427-460) */
    auto props = [&](int k, int j, double &s_, double &m_, double &w_) {
        const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
        if (a.grad && (itf.energy_n || itf.mobility_n)) {
            double u[3], nrm = 0.0;
            for (int d = 0; d < DIM; d++) {
                u[d] = a.grad[((int64_t)d * a.P + k) * S + c] - a.grad[((int64_t)d * a.P + j) * S + c];
                nrm += u[d] * u[d];
            }
            nrm = sqrt(nrm);
            if (nrm > 1e-16)
                for (int d = 0; d < DIM; d++) u[d] /= nrm;
            interface_props_aniso(itf, T, u, DIM, s_, m_, w_);
        } else {
            interface_props(itf, T, s_, m_, w_);
        }
    };
    for (int g = 0; g < PM; g++) pf[g] = 0.0;
    /* the interface terms (capillary force, active set, constrained rates)
     * in the compute type RC: FP64 on the FP64 path (the reference's
     * operations), FP32 on the mixed path; the chemical driving force comes
     * from the FP64 model evaluation above */
    auto interface_rates = [&](auto zero) {
        using RC = decltype(zero);
        const RC PIc = (RC)PI;
        RC cap[PM], unc[PM], rate[PM];
        for (int g = 0; g < n; g++) { cap[g] = (RC)0; rate[g] = (RC)0; }
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                double skd, mkd, wkd;
                props(k, j, skd, mkd, wkd);
                const RC skj = (RC)skd, wkj = (RC)wkd;
                cap[k] -= skj * ((RC)phi[j] / wkj + (RC)lap[j] * wkj / PIc / PIc);
                cap[j] -= skj * ((RC)phi[k] / wkj + (RC)lap[k] * wkj / PIc / PIc);
                for (int i = j + 1; i < n; i++) {
                    double s_, m_, w_;
                    RC tj = (RC)0, v;
                    v = skj / wkj; tj = tj > v ? tj : v;
                    props(k, i, s_, m_, w_);
                    v = (RC)s_ / (RC)w_; tj = tj > v ? tj : v;
                    props(j, i, s_, m_, w_);
                    v = (RC)s_ / (RC)w_; tj = tj > v ? tj : v;
                    tj *= (RC)a.junctionpenalty;
                    cap[k] -= tj * (RC)phi[j] * (RC)phi[i];
                    cap[j] -= tj * (RC)phi[k] * (RC)phi[i];
                    cap[i] -= tj * (RC)phi[k] * (RC)phi[j];
                }
            }
            cap[k] *= (RC)8;
            cap[k] += (RC)lap[k];
        }
        /* chemical driving force (src/cipher.c:499-522) */
        for (int k = 0; k < n; k++)
            for (int j = k + 1; j < n; j++) {
                const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
                if (itf.has_potential) {
                    double v = 0.0;
                    for (int d = 0; d < ndp; d++) v += itf.potential[d] * cbar[d];
                    chem[k] += v * h[j];
                    chem[j] += v * h[k];
                }
            }
        interpolant_dT<PM>(a.interp, chem, phi, n);
        /* active set and constrained rate (src/cipher.c:524-555) */
        RC nact = (RC)0;
        uint32_t act = 0;
        for (int g = 0; g < n; g++) unc[g] = (RC)0;
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                double s_, m_, w_;
                props(k, j, s_, m_, w_);
                const RC r = (RC)m_ * ((cap[k] - cap[j]) - (RC)(chem[k] - chem[j]) * (RC)8 * (RC)sqrt(h[k] * h[j]) / PIc);
                unc[k] += r;
                unc[j] -= r;
            }
            const bool on = (phi[k] > CIPHER_TOL && phi[k] < 1.0 - CIPHER_TOL) || (phi[k] < CIPHER_TOL && unc[k] > (RC)0) ||
                            (phi[k] > 1.0 - CIPHER_TOL && unc[k] < (RC)0);
            if (on) { act |= 1u << k; nact += (RC)1; }
        }
        for (int k = 0; k < n; k++) {
            if (!(act >> k & 1u)) continue;
            for (int j = k + 1; j < n; j++) {
                if (!(act >> j & 1u)) continue;
                double s_, m_, w_;
                props(k, j, s_, m_, w_);
                const RC r = (RC)m_ * ((cap[k] - cap[j]) - (RC)(chem[k] - chem[j]) * (RC)8 * (RC)sqrt(h[k] * h[j]) / PIc);
                rate[k] += r;
                rate[j] -= r;
            }
            rate[k] /= nact;
        }
        for (int g = 0; g < n; g++) pf[g] = (double)rate[g];
    };
    if (n > 1) {
        if constexpr (sizeof(R) == 4) interface_rates(0.0f);
        else interface_rates(0.0);
    }
    for (int g = 0; g < a.P; g++) a.fphi[(int64_t)g * S + c] = (R)(g < PM ? pf[g] : 0.0);

    /* temperature rate (src/cipher.c:558-568) */
    double cp = 0.0, tr = ltm;
    for (int g = 0; g < n; g++) {
        const cipher_material &mat = material_of(ch, ids[g]);
        if (mat.specific_heat.n) cp += h[g] * tseries(T, mat.specific_heat);
        if (mat.latent_heat.n) tr += pf[g] * tseries(T, mat.latent_heat);
    }
    if (cp != 0.0) tr /= cp;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = (R)tr;

    if (!ndp) return;
    /* composition rate and dmu/dt (src/cipher.c:583-662) */
    const int DN = CIPHER_MAXCP - 1;
    double cpv[PM * (CIPHER_MAXCP - 1)];
    for (int q = 0; q < n * DN; q++) cpv[q] = 0.0;
    for (int k = 0; k < n; k++)
        for (int j = k + 1; j < n; j++) {
            const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
            if (itf.has_potential)
                for (int d = 0; d < ndp; d++) {
                    cpv[k * DN + d] += itf.potential[d] * h[j];
                    cpv[j * DN + d] += itf.potential[d] * h[k];
                }
        }
    for (int g = 0; g < n; g++) {
        double tmp[CIPHER_MAXCP];
        for (int d = 0; d < ndp; d++) tmp[d] = cpv[g * DN + d];
        matvec(&cpv[g * DN], dcdm, tmp, ndp);
    }
    double wdp[CIPHER_MAXCP];
    for (int d = 0; d < CIPHER_MAXCP; d++) wdp[d] = 0.0;
    if (n > 1) {
        for (int d = 0; d < ndp; d++) {
            double wpf[PM];
            for (int g = 0; g < n; g++) wpf[g] = yw[g * DN + d] - cpv[g * DN + d];
            interpolant_dT<PM>(a.interp, wpf, phi, n);
            for (int g = 0; g < n; g++) wdp[d] -= pf[g] * wpf[g];
        }
    }
    /* solute sources (material.c:295-351; sink model) */
    double src[CIPHER_MAXCP], comp[CIPHER_MAXCP];
    for (int d = 0; d < ncp; d++) { src[d] = 0.0; comp[d] = a.comp[(int64_t)d * S + c]; }
    for (int k = 0; k < n; k++) {
        const cipher_material &mat = material_of(ch, ids[k]);
        for (int s = 0; s < mat.nsources; s++) {
            double tmp[CIPHER_MAXCP];
            for (int d = 0; d < ncp; d++) tmp[d] = mat.sources[s].rate[d] * (mat.sources[s].ceq[d] - comp[d]);
            for (int d = 0; d < ncp; d++) src[d] += h[k] * h[k] * tmp[d];
        }
        for (int j = k + 1; j < n; j++) {
            const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
            for (int s = 0; s < itf.nsources; s++) {
                double tmp[CIPHER_MAXCP];
                for (int d = 0; d < ncp; d++) tmp[d] = itf.sources[s].rate[d] * (itf.sources[s].ceq[d] - comp[d]);
                for (int d = 0; d < ncp; d++) src[d] += 2.0 * h[k] * h[j] * tmp[d];
            }
        }
    }
    for (int d = 0; d < ndp; d++) wdp[d] += (ldp[d] + src[d]);
    for (int g = 0; g < n; g++) {
        const cipher_material &mat = material_of(ch, ids[g]);
        if (n > 1) {
            double pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP];
            slot_potential(a, mat, mu, ci, c, g, pot);
            sitefrac(ch, ids[g], pot, T, y);
            sitefrac_tangent(ch, ids[g], y, pot, T, tpot, tex, tT);
        }
        for (int s = 0; s < mat.nsites; s++) {
            double dex[CIPHER_MAXCP];
            for (int d = 0; d < ndp; d++) dex[d] = a.fex[(int64_t)(g * SP + s * ndp + d) * S + c];
            matvec(&cpv[g * DN], &tex[s * ndp * ndp], dex, ndp);
            for (int d = 0; d < ndp; d++)
                wdp[d] -= h[g] * mat.stoichiometry[s] * (cpv[g * DN + d] + tT[s * ndp + d] * tr);
        }
    }
    double dmdc[(CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1)], out[CIPHER_MAXCP];
    invert_small(dmdc, dcdm, ndp);
    matvec(out, dmdc, wdp, ndp);
    for (int d = 0; d < ndp; d++) a.fdp[(int64_t)d * S + c] = out[d];
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
 * temperature keep reading the original. */
template <typename R>
__global__ void __launch_bounds__(256) k_specialise(const cipher_material *mat, cipher_material *spec, const R *tm,
                                                    double *tspec)
{
    const double T = (double)tm[0];
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
    if (blockIdx.x == 0 && threadIdx.x == 0) *tspec = T;
}

/* ------------------------------------------------------------------ */
/* launchers                                                            */
/* ------------------------------------------------------------------ */

template <typename R>
static cudaError_t launch_gen(const GenArgs<R> &a, int dim, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((a.ncells + kGenBlock - 1) / kGenBlock);
    if (a.chem.spec)
        k_specialise<R><<<a.chem.nmat, 256, 0, s>>>(a.chem.mat, (cipher_material *)a.chem.spec, a.tm,
                                                     (double *)a.chem.tspec);
    if (a.order) {
        const OrderBuf o = {a.order, a.order_counts, a.order_cursor, a.nclass, a.ncells};
        launch_order(o, GeneralClassKey{a.as, a.stride, a.chem.pmm, a.npf, a.chem.nmat}, s);
    }
    if (a.ndp) k_chem_cell<CIPHER_PMAX, R><<<blocks, kGenBlock, 0, s>>>(a);
    if (a.grad) k_gradients<CIPHER_PMAX, R><<<blocks, kGenBlock, 0, s>>>(a, dim);
    k_rhs_general<CIPHER_PMAX, R><<<blocks, kGenBlock, 0, s>>>(a, dim);
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
