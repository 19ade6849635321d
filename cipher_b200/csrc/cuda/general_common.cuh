/*
 * general_common.cuh - per-cell pieces shared by the general (chemistry)
 * RHS kernels: the interpolant, segregation and site potentials, set
 * loading, the reference's face order and face divisor, the walk over a
 * cell's faces, the chemical-potential and heat fluxes of one face, the
 * boundary faces, and the cell classes of the grouping.
 *
 * Every helper is force-inlined and takes the component count NC as a
 * template argument (0: read from the arguments), so a kernel compiled for
 * one NC keeps its per-component arrays in registers; NC = 0 and NC > 0 run
 * the same operations in the same order and give the same bits.  Only units
 * compiled with --fmad=false include this header.
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "kernels.h"
#include "models.cuh"

namespace cipher {

constexpr int kGenBlock = 128;
/* one warp per block for the kernels whose work sits in few cells (the
 * cells of several phases, clustered where the grouping puts them): the
 * block scheduler then spreads those warps over all SMs */
constexpr int kWarpBlock = 32;
/* the single-phase and item kernels serve contexts of more cells than this */
constexpr int64_t kSpecialisedMinCells = 16384;

/* phase interpolant h and its transposed derivative (src/utility.c:470-557) */
__device__ __forceinline__ void interpolant(int kind, const double *phi, int n, double *h)
{
    if (kind == CIPHER_INTERP_LINEAR) {
#pragma unroll
        for (int g = 0; g < n; g++) h[g] = phi[g];
        return;
    }
    if (n == 1) { h[0] = 1.0; return; }
    double sum = 0.0;
#pragma unroll
    for (int g = 0; g < n; g++) {
        h[g] = kind == CIPHER_INTERP_QUADRATIC ? phi[g] * phi[g] : phi[g] * phi[g] * (3.0 - 2.0 * phi[g]);
        sum += h[g];
    }
#pragma unroll
    for (int g = 0; g < n; g++) h[g] /= sum;
}

template <int PM>
__device__ __forceinline__ void interpolant_dT(int kind, double *v, const double *phi, int n)
{
    if (kind == CIPHER_INTERP_LINEAR) return;
    if (n == 1) { v[0] = 0.0; return; }
    double avg = 0.0, sum = 0.0;
#pragma unroll
    for (int g = 0; g < n; g++) {
        double w = kind == CIPHER_INTERP_QUADRATIC ? phi[g] * phi[g] : phi[g] * phi[g] * (3.0 - 2.0 * phi[g]);
        sum += w;
        avg += w * v[g];
    }
#pragma unroll
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
template <int NC = 0, int MODEL = -1, typename R>
__device__ __forceinline__ void slot_potential(const GenArgs<R> &a, const cipher_material &mat, const double *mu,
                                               const double *ci, int64_t c, int g, double *pot)
{
    const int64_t S = a.stride;
    const int ndp = NC > 0 ? NC - 1 : a.ndp;
#pragma unroll
    for (int s = 0; s < PhaseModel<NC, MODEL>::nsites(mat); s++) {
#pragma unroll
        for (int d = 0; d < ndp; d++)
            pot[s * ndp + d] = mat.stoichiometry[s] * (mu[d] - ci[d]) -
                               a.ex[(int64_t)(g * a.SP + s * ndp + d) * S + c];
    }
}

/* segregation potential of the cell, sum_{k<j} h_k h_j V_kj (src/cipher.c:160-172) */
template <int NC = 0, typename R>
__device__ __forceinline__ void segregation(const GenArgs<R> &a, const uint16_t *ids, const double *h, int n,
                                            double *ci)
{
    const int ndp = NC > 0 ? NC - 1 : a.ndp;
#pragma unroll
    for (int d = 0; d < CIPHER_MAXCP; d++) ci[d] = 0.0;
#pragma unroll
    for (int k = 0; k < n; k++) {
#pragma unroll
        for (int j = k + 1; j < n; j++) {
            const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
            if (itf.has_potential) {
#pragma unroll
                for (int d = 0; d < ndp; d++) ci[d] += h[k] * h[j] * itf.potential[d];
            }
        }
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
#pragma unroll
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
/* cell classes of the grouping                                         */
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


/* neighbour at face position f in the reference's face order: [0,DIM)
 * below without wrap (descending d), [DIM,2DIM) own faces (ascending d),
 * [2DIM,3DIM) wrapped around from above (ascending d); -1 if absent */
__device__ __forceinline__ int64_t gen_face_nb(const int *res, const int *per, int64_t c, const int *co, int f,
                                               const int DIM)
{
    /* the axis-indexed values as selects rather than indexed arrays, so that
     * they stay in registers (a runtime index would place them in local
     * memory) */
    auto sel3 = [](const int *v, int d) { return d == 0 ? v[0] : d == 1 ? v[1] : v[2]; };
    const int64_t r0 = res[0], r01 = (int64_t)res[0] * res[1];
    auto st = [&](int d) -> int64_t { return d == 0 ? 1 : d == 1 ? r0 : r01; };
    if (f < DIM) {
        const int e = DIM - 1 - f;
        return sel3(co, e) > 0 ? c - st(e) : -1;
    }
    if (f < 2 * DIM) {
        const int d = f - DIM, rd = sel3(res, d);
        if (sel3(co, d) < rd - 1) return c + st(d);
        return (sel3(per, d) && rd > 1) ? c - (int64_t)(rd - 1) * st(d) : -1;
    }
    const int d = f - 2 * DIM, rd = sel3(res, d);
    return (sel3(co, d) == 0 && sel3(per, d) && rd > 1) ? c + (int64_t)(rd - 1) * st(d) : -1;
}

/* ff*x/vol as the reference forms it (src/cipher.c:281-282) */
template <typename R>
__device__ __forceinline__ double face_div(const GenArgs<R> &a, double x)
{
    if (a.geom_mode == 2) return x;
    if (a.geom_mode == 1) return (a.ffactor * x) * a.inv_vol;
    return (a.ffactor * x) / a.vol;
}

/* ------------------------------------------------------------------ */
/* faces                                                                */
/* ------------------------------------------------------------------ */

/* the faces of cell c in the reference's face order (src/cipher.c:235-317):
 * visit(nb, self_L, nn, fdiv) for each face whose other cell nb holds a
 * valid set of nn phases (a cell with an invalid set raises the flag from
 * its own thread); fdiv(x) = ff*x/vol of cell c as the reference forms it
 * (src/cipher.c:281-282).  co: the cell's grid coordinates (uniform grid). */
template <typename R, typename Visit>
__device__ __forceinline__ void walk_faces(const GenArgs<R> &a, int64_t c, const int *co, const int DIM,
                                           Visit &&visit)
{
    const bool listed = a.fl.start != nullptr;   /* an adapted mesh: faces from the lists */
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
        auto fdiv = [&](double x) { return listed ? (ffv * x) / vol_c : face_div(a, x); };
        const int nn = a.as[nb];
        if (nn < 1 || nn > a.P) continue;
        visit(nb, self_L, nn, fdiv);
    }
}

/* chemical-potential flux with the Andersson-Agren frame (material.c:
 * 1125-1137) and heat flux of the face between cl and cr, added to
 * (self_L) or subtracted from the cell's divergences ldp and ltm.  Mixed
 * layout (R = float): the flux stencil in FP32 - the Andersson-Agren matrix
 * and its product with the potential difference (formed in FP64, then
 * rounded) - and the heat-flux product in FP32, each face flux summed into
 * the FP64 divergence. */
template <int NC, typename R, typename Div>
__device__ __forceinline__ void chem_heat_face(const GenArgs<R> &a, int64_t cl, int64_t cr, bool self_L,
                                               const Div &fdiv, double *ldp, double &ltm)
{
    const int64_t S = a.stride;
    const int ncp = NC > 0 ? NC : a.ncp, ndp = NC > 0 ? NC - 1 : a.ndp;
    if (ndp) {
        double me[CIPHER_MAXCP], ca[CIPHER_MAXCP];
#pragma unroll
        for (int d = 0; d < ncp; d++) {
            const double ml = a.mob[(int64_t)d * S + cl], mr = a.mob[(int64_t)d * S + cr];
            const double cL = a.comp[(int64_t)d * S + cl], cR = a.comp[(int64_t)d * S + cr];
            if (fabs(ml) > 1e-32 && fabs(mr) > 1e-32) me[d] = 2.0 * ml * mr / (ml + mr);
            else me[d] = 0.0;
            ca[d] = 2.0 * cL * cR / (cL + cR);
        }
        if constexpr (sizeof(R) == 4) {
            float MB[(CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1)], dmu[CIPHER_MAXCP];
#pragma unroll
            for (int i = 0; i < ndp; i++) {
#pragma unroll
                for (int j = 0; j < ndp; j++) {
                    float acc = 0.0f;
#pragma unroll
                    for (int k = 0; k < ncp; k++)
                        acc += ((j == k ? 1.0f : 0.0f) - (float)ca[j]) * ((k == i ? 1.0f : 0.0f) - (float)ca[i]) *
                               (float)me[k];
                    MB[i * ndp + j] = acc;
                }
            }
#pragma unroll
            for (int d = 0; d < ndp; d++) dmu[d] = (float)(a.dp[(int64_t)d * S + cr] - a.dp[(int64_t)d * S + cl]);
#pragma unroll
            for (int d = 0; d < ndp; d++) {
                float f = 0.0f;
#pragma unroll
                for (int j = 0; j < ndp; j++) f += MB[d * ndp + j] * dmu[j];
                if (self_L) ldp[d] += fdiv((double)f);
                else ldp[d] -= fdiv((double)f);
            }
        } else {
            double MB[(CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1)], dmu[CIPHER_MAXCP], fl[CIPHER_MAXCP];
#pragma unroll
            for (int i = 0; i < ndp; i++) {
#pragma unroll
                for (int j = 0; j < ndp; j++) {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < ncp; k++)
                        acc += ((j == k ? 1.0 : 0.0) - ca[j]) * ((k == i ? 1.0 : 0.0) - ca[i]) * me[k];
                    MB[i * ndp + j] = acc;
                }
            }
#pragma unroll
            for (int d = 0; d < ndp; d++) dmu[d] = a.dp[(int64_t)d * S + cr] - a.dp[(int64_t)d * S + cl];
            matvec(fl, MB, dmu, ndp);
#pragma unroll
            for (int d = 0; d < ndp; d++) {
                if (self_L) ldp[d] += fdiv(fl[d]);
                else ldp[d] -= fdiv(fl[d]);
            }
        }
    }
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

/* boundary faces of cell c (src/cipher.c:319-389): the conditions in
 * their order, each over the cell's faces on the domain boundary */
template <int NC, typename R>
__device__ __forceinline__ void boundary_faces(const GenArgs<R> &a, int64_t c, const int *co, const int DIM, double T,
                                               const double *mu, double *ldp, double &ltm)
{
    if (!a.nbcs) return;
    const int64_t S = a.stride;
    const int ndp = NC > 0 ? NC - 1 : a.ndp;
    const bool listed = a.fl.start != nullptr;
    const double dc = listed ? a.fl.delta[c] : a.delta;
    const double cf = 1.0 / ipow(dc, 2);
    const double tcc = a.tcond ? a.tcond[c] : 0.0;
    const int q0 = listed ? a.fl.bstart[c] : 0, q1 = listed ? a.fl.bstart[c + 1] : 2 * DIM;
#pragma unroll
    for (int b = 0; b < CIPHER_MAXBC; b++) {
        if (b >= a.nbcs) break;
        const DevBC &bc = a.bcs[b];
#pragma unroll 1
        for (int q = q0; q < q1; q++) {
            if (listed) {
                if (bc.label != a.fl.blabel[q]) continue;
            } else {
                const int d = q >> 1;
                const int per_d = d == 0 ? a.per[0] : d == 1 ? a.per[1] : a.per[2];
                const int res_d = d == 0 ? a.res[0] : d == 1 ? a.res[1] : a.res[2];
                const int co_d = d == 0 ? co[0] : d == 1 ? co[1] : co[2];
                if (per_d) continue;
                const bool on = (q & 1) ? co_d == res_d - 1 : co_d == 0;
                if (!on || bc.label != 2 * d + 1 + (q & 1)) continue;
            }
            double fd[CIPHER_MAXCP];
#pragma unroll
            for (int k = 0; k < CIPHER_MAXCP; k++) fd[k] = 0.0;
            if (bc.chem_type != CIPHER_BC_NONE) {
                if (bc.chem_type == CIPHER_BC_NEUMANN) {
#pragma unroll
                    for (int k = 0; k < ndp; k++) if (bc.chem_on[k]) fd[k] = bc.chem_val[k] * dc;
                } else {
#pragma unroll
                    for (int k = 0; k < ndp; k++)
                        if (bc.chem_on[k]) fd[k] = a.mob[(int64_t)k * S + c] * (bc.chem_val[k] - mu[k]);
                }
            }
            double fluxt = 0.0;
            if (bc.thermal_type == CIPHER_BC_NEUMANN) fluxt = tcc * bc.thermal_val * dc;
            else if (bc.thermal_type == CIPHER_BC_DIRICHLET) fluxt = tcc * (bc.thermal_val - T);
            if (bc.chem_type != CIPHER_BC_NONE) {
#pragma unroll
                for (int k = 0; k < ndp; k++) ldp[k] += cf * fd[k];
            }
            if (bc.thermal_type != CIPHER_BC_NONE) ltm += cf * fluxt;
        }
    }
}

/* ------------------------------------------------------------------ */
/* single-phase cells evaluated by kernels of their own                 */
/* ------------------------------------------------------------------ */

/* the model of cell c when the cell holds one phase whose material's model
 * has a kernel of its own (bit `model` of a.single_models, rhs_single.cu),
 * else -1 */
template <typename R>
__device__ __forceinline__ int single_model(const GenArgs<R> &a, int64_t c)
{
    if (!a.single_models || a.as[c] != 1) return -1;
    const int id = a.as[a.stride + c];
    if (id >= a.npf) return -1;
    const int m = a.chem.pmm[id];
    if (m < 0 || m >= a.chem.nmat) return -1;
    const int model = a.chem.mat[m].model;
    return (model >= 0 && model < 32 && (a.single_models >> model & 1u)) ? model : -1;
}

/* ------------------------------------------------------------------ */
/* (cell, phase) items of the cells of several phases                   */
/* ------------------------------------------------------------------ */

/* per item, the model results the general kernels combine (rhs_items.cu
 * writes them): the phase's chemical energy, its weighted site fractions
 * yw[d] = sum_s stoichiometry_s y_s,d, its site fractions y[s][d] (d < ndp),
 * the tangent blocks tpot[s], tex[s] (ndp x ndp) and tT[s] (ndp), for s
 * below the largest sublattice count, and for the cell's composition and
 * mobility (k_chem_cell) its site fractions of every component yc[s][d]
 * (d < ncp = ndp + 1) and its component mobilities me[d]; stored as planes
 * q of icap items */
struct ItemQ {
    int yw, y, tpot, tex, tt, yc, me, nq;
};

__host__ __device__ inline ItemQ item_q(int ndp, int SP)
{
    const int ns = ndp ? SP / ndp : 0;
    ItemQ q;
    q.yw = 1;
    q.y = q.yw + ndp;
    q.tpot = q.y + ns * ndp;
    q.tex = q.tpot + ns * ndp * ndp;
    q.tt = q.tex + ns * ndp * ndp;
    q.yc = q.tt + ns * ndp;
    q.me = q.yc + ns * (ndp + 1);
    q.nq = q.me + (ndp + 1);
    return q;
}

}  // namespace cipher
