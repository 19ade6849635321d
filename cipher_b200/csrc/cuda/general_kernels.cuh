/*
 * general_kernels.cuh - the per-cell general (chemistry) kernels: every
 * cell that the single-phase kernels (rhs_single.cu) do not take, any set
 * size, component count and mix of models.
 *
 * A cell of several phases whose phases were evaluated by the item kernel
 * (rhs_items.cu: one thread per phase, a.ibase[c] >= 0) reads each phase's
 * energy, site fractions, tangent and explicit-potential rates from the
 * item scratch instead of evaluating the models here; the arithmetic that
 * combines them is the same, in the same order, so the results are the
 * same bits.  The model chains of a cell of n phases then run on n threads
 * in parallel instead of one after the other on one thread.
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "general_common.cuh"
#include "kernels.h"
#include "models.cuh"

namespace cipher {

/* ------------------------------------------------------------------ */
/* per-cell composition, mobility and conductivity                      */
/* ------------------------------------------------------------------ */

template <int PM, typename R>
__global__ void __launch_bounds__(kWarpBlock) k_chem_cell(const GenArgs<R> a)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ncells) return;
    const int64_t c = a.order ? (int64_t)a.order[t] : t;
    if (single_model(a, c) >= 0) return;           /* rhs_single.cu's kernels */
    const int64_t S = a.stride;
    const int ncp = a.ncp, ndp = a.ndp;
    uint16_t ids[PM];
    double phi[PM], h[PM];
    const int n = load_set<PM>(a, c, ids, phi);
    /* >= 0: the phases' site fractions and mobilities are items ib .. ib+n-1 */
    const int32_t ib = a.ibase ? a.ibase[c] : -1;
    const ItemQ iq = item_q(ndp, a.SP);
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
            if (ib >= 0) {
                const int64_t it = (int64_t)ib + g;
                for (int d = 0; d < ncp; d++) me[d] = a.iscr[(int64_t)(iq.me + d) * a.icap + it];
                for (int s = 0; s < mat.nsites; s++)
                    for (int d = 0; d < ncp; d++)
                        y[s * ncp + d] = a.iscr[(int64_t)(iq.yc + s * ncp + d) * a.icap + it];
            } else {
                slot_potential(a, mat, mu, ci, c, g, pot);
                sitefrac(ch, ids[g], pot, T, y);
                mobility(ch, ids[g], y, T, me);
            }
            for (int d = 0; d < ncp; d++) mm[d] += h[g] * me[d];
            for (int s = 0; s < mat.nsites; s++) {
                for (int d = 0; d < ncp; d++) cc[d] += h[g] * mat.stoichiometry[s] * y[s * ncp + d];
            }
            if (mat.tconductivity.n) tc += h[g] * tseries(T, mat.tconductivity);
        }
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
                if (itf.has_mobilityc) {
                    for (int d = 0; d < ncp; d++) mm[d] *= exp(itf.mobilityc[d] / CIPHER_R_GAS / T);
                }
            }
        }
    }
    for (int d = 0; d < ncp; d++) {
        a.comp[(int64_t)d * S + c] = cc[d];
        a.mob[(int64_t)d * S + c] = mm[d];
    }
    a.tcond[c] = tc;
}

/* ------------------------------------------------------------------ */
/* the RHS                                                              */
/* ------------------------------------------------------------------ */

/* two warps per 32 cells (one warp's worth of cells per block): the first
 * gathers the faces (phase, mu and heat fluxes, boundary faces) while the
 * second runs the cell terms that do not depend on them (interpolant,
 * segregation, the pass over the phases); the face sums then pass to the
 * second warp through shared memory.  The operations are the same. */
template <int PM, typename R>
__global__ void __launch_bounds__(2 * kWarpBlock, 16) k_rhs_general(const GenArgs<R> a, const int DIM)
{
    __shared__ double sh_lap[PM][kWarpBlock], sh_ldp[CIPHER_MAXCP][kWarpBlock], sh_ltm[kWarpBlock];
    const int lane = threadIdx.x & 31;
    const bool face_warp = threadIdx.x < kWarpBlock;
    const int64_t t = (int64_t)blockIdx.x * kWarpBlock + lane;
    bool active = t < a.ncells;
    const int64_t c = active ? (a.order ? (int64_t)a.order[t] : t) : 0;
    if (active && single_model(a, c) >= 0) active = false;   /* rhs_single.cu's kernels */
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
    const int n = active ? load_set<PM>(a, c, ids, phi) : 0;
    if (n == 0) active = false;
    /* >= 0: the phases' model results are items ib .. ib+n-1 of the scratch */
    const int32_t ib = active && a.ibase ? a.ibase[c] : -1;
    const ItemQ iq = item_q(ndp, SP);
    auto item = [&](int q, int g) { return a.iscr[(int64_t)q * a.icap + ib + g]; };
    const double T = active ? (double)a.tm[c] : 0.0;
    const ChemTables ch = chem_at(a.chem, T);
    double mu[CIPHER_MAXCP], ldp[CIPHER_MAXCP];
    for (int d = 0; d < ndp; d++) { mu[d] = active ? a.dp[(int64_t)d * S + c] : 0.0; ldp[d] = 0.0; }
    double ltm = 0.0;
    for (int g = 0; g < n; g++) lap[g] = 0.0;

    if (active && face_warp) {
        /* ---- faces in the reference's face order (src/cipher.c:235-317) ---- */
        walk_faces(a, c, co, DIM, [&](int64_t nb, bool self_L, int nn, const auto &fdiv) {
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
            const int64_t cl = self_L ? c : nb, cr = self_L ? nb : c;
            chem_heat_face<0>(a, cl, cr, self_L, fdiv, ldp, ltm);
        });
        boundary_faces<0>(a, c, co, DIM, T, mu, ldp, ltm);
        for (int g = 0; g < n; g++) sh_lap[g][lane] = lap[g];
        for (int d = 0; d < ndp; d++) sh_ldp[d][lane] = ldp[d];
        sh_ltm[lane] = ltm;
    }

    double ci[CIPHER_MAXCP];
    double chem[PM], yw[PM * (CIPHER_MAXCP - 1)];
    double cbar[CIPHER_MAXCP], dcdm[(CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1)];
    /* tangent of the last phase evaluated: reused by the composition rate
     * below when the cell has a single phase (same arguments, same bits) */
    double tpot[2 * 16], tex[2 * 16], tT[2 * CIPHER_MAXCP];
    if (active && !face_warp) {
        /* ---- cell terms (src/cipher.c:391-664) ---- */
        interpolant(a.interp, phi, n, h);
        if (ndp) segregation(a, ids, h, n, ci);

        /* pass over the phases: driving force, dEX/dt and the tangent sum */
        for (int d = 0; d < CIPHER_MAXCP; d++) cbar[d] = 0.0;
        for (int q = 0; q < (CIPHER_MAXCP - 1) * (CIPHER_MAXCP - 1); q++) dcdm[q] = 0.0;
        for (int g = 0; g < n; g++) {
            const cipher_material &mat = material_of(ch, ids[g]);
            if (ib >= 0) {
                /* the same sums over the item's stored results (n > 1, ndp > 0) */
                chem[g] = item(0, g);
                for (int s = 0; s < mat.nsites; s++)
                    for (int d = 0; d < ndp; d++) cbar[d] += h[g] * mat.stoichiometry[s] * item(iq.y + s * ndp + d, g);
                for (int d = 0; d < ndp; d++) yw[g * (CIPHER_MAXCP - 1) + d] = item(iq.yw + d, g);
                for (int s = 0; s < mat.nsites; s++)
                    for (int q = 0; q < ndp * ndp; q++)
                        dcdm[q] += h[g] * mat.stoichiometry[s] * mat.stoichiometry[s] * item(iq.tpot + s * ndp * ndp + q, g);
                continue;
            }
            double pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP];
            if (ndp) {
                slot_potential(a, mat, mu, ci, c, g, pot);
                sitefrac(ch, ids[g], pot, T, y);
            }
            if (n > 1) {
                chem[g] = chemenergy(ch, ids[g], y, mu, T);
                for (int s = 0; s < mat.nsites; s++) {
                    for (int d = 0; d < ndp; d++) cbar[d] += h[g] * mat.stoichiometry[s] * y[s * ncp + d];
                }
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
                for (int s = 0; s < mat.nsites; s++) {
                    for (int d = 0; d < ndp; d++) {
                        const int64_t pl = (int64_t)(g * SP + s * ndp + d) * S + c;
                        a.fex[pl] = mat.chempot_ex_kineticcoeff * (spx[s * ndp + d] - a.ex[pl]);
                    }
                }
                for (int q = mat.nsites * ndp; q < SP; q++) a.fex[(int64_t)(g * SP + q) * S + c] = 0.0;
                sitefrac_tangent(ch, ids[g], y, pot, T, tpot, tex, tT);
                for (int s = 0; s < mat.nsites; s++) {
                    for (int q = 0; q < ndp * ndp; q++)
                        dcdm[q] += h[g] * mat.stoichiometry[s] * mat.stoichiometry[s] * tpot[s * ndp * ndp + q];
                }
            }
        }
        for (int q = n * SP; q < a.P * SP; q++) a.fex[(int64_t)q * S + c] = 0.0;
    }
    __syncthreads();
    if (!active || face_warp) return;
    for (int g = 0; g < n; g++) lap[g] = sh_lap[g][lane];
    for (int d = 0; d < ndp; d++) ldp[d] = sh_ldp[d][lane];
    ltm = sh_ltm[lane];

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
        /* the pair properties once per pair, as the reference forms them
         * (src/cipher.c:420-472), for the capillary, triple-junction,
         * active-set and rate terms below */
        double psig[PM * (PM - 1) / 2], pmob[PM * (PM - 1) / 2], pwid[PM * (PM - 1) / 2];
        auto pi = [&](int k, int j) { return k * (2 * n - k - 1) / 2 + (j - k - 1); };
        for (int k = 0; k < n; k++)
            for (int j = k + 1; j < n; j++) props(k, j, psig[pi(k, j)], pmob[pi(k, j)], pwid[pi(k, j)]);
        for (int g = 0; g < n; g++) { cap[g] = (RC)0; rate[g] = (RC)0; }
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                const RC skj = (RC)psig[pi(k, j)], wkj = (RC)pwid[pi(k, j)];
                cap[k] -= skj * ((RC)phi[j] / wkj + (RC)lap[j] * wkj / PIc / PIc);
                cap[j] -= skj * ((RC)phi[k] / wkj + (RC)lap[k] * wkj / PIc / PIc);
                for (int i = j + 1; i < n; i++) {
                    RC tj = (RC)0, v;
                    v = skj / wkj; tj = tj > v ? tj : v;
                    v = (RC)psig[pi(k, i)] / (RC)pwid[pi(k, i)]; tj = tj > v ? tj : v;
                    v = (RC)psig[pi(j, i)] / (RC)pwid[pi(j, i)]; tj = tj > v ? tj : v;
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
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
                if (itf.has_potential) {
                    double v = 0.0;
                    for (int d = 0; d < ndp; d++) v += itf.potential[d] * cbar[d];
                    chem[k] += v * h[j];
                    chem[j] += v * h[k];
                }
            }
        }
        interpolant_dT<PM>(a.interp, chem, phi, n);
        /* active set and constrained rate (src/cipher.c:524-555) */
        RC nact = (RC)0;
        uint32_t act = 0;
        for (int g = 0; g < n; g++) unc[g] = (RC)0;
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                const RC r = (RC)pmob[pi(k, j)] *
                             ((cap[k] - cap[j]) - (RC)(chem[k] - chem[j]) * (RC)8 * (RC)sqrt(h[k] * h[j]) / PIc);
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
                const RC r = (RC)pmob[pi(k, j)] *
                             ((cap[k] - cap[j]) - (RC)(chem[k] - chem[j]) * (RC)8 * (RC)sqrt(h[k] * h[j]) / PIc);
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
    for (int g = 0; g < PM; g++)
        if (g < a.P) a.fphi[(int64_t)g * S + c] = (R)pf[g];
    for (int g = PM; g < a.P; g++) a.fphi[(int64_t)g * S + c] = (R)0.0;

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
    for (int k = 0; k < n; k++) {
        for (int j = k + 1; j < n; j++) {
            const DevInterface &itf = pair_itf(a, ids[k], ids[j]);
            if (itf.has_potential) {
                for (int d = 0; d < ndp; d++) {
                    cpv[k * DN + d] += itf.potential[d] * h[j];
                    cpv[j * DN + d] += itf.potential[d] * h[k];
                }
            }
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
        if (ib >= 0) {
            for (int q = 0; q < mat.nsites * ndp * ndp; q++) tex[q] = item(iq.tex + q, g);
            for (int q = 0; q < mat.nsites * ndp; q++) tT[q] = item(iq.tt + q, g);
        } else if (n > 1) {
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

}  // namespace cipher
