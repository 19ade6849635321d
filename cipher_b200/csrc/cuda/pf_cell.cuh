/*
 * pf_cell.cuh - cell terms of the phase-field RHS in the reference's
 * operation order (src/cipher.c:417-555): capillary force with the
 * triple-junction penalty, the unconstrained pair rates, the active set and
 * the constrained rate.
 *
 * The reference accumulates each slot's capillary force inside a k<j<i loop
 * nest that also updates the other slots.  Slot m receives, in order:
 *   for k < m:  -t(k,j,m) phi_k phi_j   for k < j < m   (m as the third phase)
 *               -sigma(k,m) a_k(k,m)                     (m as the second)
 *               -t(k,m,i) phi_k phi_i   for i > m        (m as the second)
 *   for j > m:  -sigma(m,j) a_j(m,j), then -t(m,j,i) phi_j phi_i for i > j
 *   then        *8, + lap_m
 * with a_j(p,q) = phi_j/w(p,q) + lap_j*w(p,q)/pi/pi.  Evaluating that
 * sequence per slot gives the same IEEE results, and each slot's chain is
 * independent.  Triple terms whose product contains a zero phase fraction
 * are exactly zero; subtracting them leaves the running value unchanged, so
 * they are skipped: the triple part costs O(n * nz^2) with nz the number of
 * non-zero phase fractions (new phases of the neighbour union start at 0).
 * The rates follow the same per-slot decomposition.
 */
#pragma once
#include <cstdint>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"

namespace cipher {

/* pair sigma, m, w of phases (ids) a<b at temperature T */
template <typename R, bool SINGLE>
__device__ __forceinline__ void pair_props(const PfArgs<R> &a, int ia, int ib, double T, R &sig, R &mob, R &wid)
{
    if (SINGLE) {
        sig = (R)a.sig0;
        mob = (R)a.mob0;
        wid = (R)a.wid0;
    } else {
        double s, m, w;
        interface_props(a.itfs[a.itflist[ia * a.npf + ib]], T, s, m, w);
        sig = (R)s;
        mob = (R)m;
        wid = (R)w;
    }
}

/* triple-junction weight of phases (ids) a<b<c (src/cipher.c:482-489) */
template <typename R, bool SINGLE>
__device__ __forceinline__ R triple_weight(const PfArgs<R> &a, int ia, int ib, int ic, double T)
{
    if (SINGLE) return (R)a.tj0;
    double s, m, w, v, t = 0.0;
    interface_props(a.itfs[a.itflist[ia * a.npf + ib]], T, s, m, w);
    v = s / w; t = t > v ? t : v;
    interface_props(a.itfs[a.itflist[ia * a.npf + ic]], T, s, m, w);
    v = s / w; t = t > v ? t : v;
    interface_props(a.itfs[a.itflist[ib * a.npf + ic]], T, s, m, w);
    v = s / w; t = t > v ? t : v;
    t *= a.junctionpenalty;
    return (R)t;
}

template <typename R, bool SINGLE>
__device__ __forceinline__ R pair_a(const SlotColumns<R> &sc, int j, R wid)
{
    if (SINGLE) return sc.AJ(j);
    const R PI = (R)CIPHER_PI_D;
    return sc.PHI(j) / wid + sc.LAP(j) * wid / PI / PI;
}

/*
 * Cell terms in reference order for a cell with n slots already gathered in
 * its columns (PHI, LAP, ID); writes all P slots of F when `live`.
 */
template <typename R, bool SINGLE>
__device__ __forceinline__ void cell_rates_ordered(const PfArgs<R> &a, const SlotColumns<R> &sc, int n, int64_t c,
                                                   bool live, double T)
{
    const int64_t S = a.stride;
    uint32_t act = 0;
    R nact = (R)0;
    if (n > 1) {
        /* non-zero phase fractions, ascending */
        int nz = 0;
        for (int g = 0; g < n; g++)
            if (sc.PHI(g) != (R)0) sc.NZ(nz++) = (uint8_t)g;
        if (SINGLE) {
            /* with one interface a_j does not depend on the pair: form it once */
            const R PI = (R)CIPHER_PI_D, wid = (R)a.wid0;
            for (int g = 0; g < n; g++) sc.AJ(g) = sc.PHI(g) / wid + sc.LAP(g) * wid / PI / PI;
        }
        /* capillary force per slot (src/cipher.c:474-497) */
        for (int m = 0; m < n; m++) {
            R cm = (R)0;
            const int idm = sc.ID(m);
            int q0 = 0;                                 /* first NZ entry > k */
            for (int k = 0; k < m; k++) {
                const R pk = sc.PHI(k);
                const int idk = sc.ID(k);
                while (q0 < nz && sc.NZ(q0) <= k) q0++;
                if (pk != (R)0) {
                    for (int q = q0; q < nz; q++) {     /* k < j < m */
                        const int j = sc.NZ(q);
                        if (j >= m) break;
                        const R t = triple_weight<R, SINGLE>(a, idk, sc.ID(j), idm, T);
                        cm -= t * pk * sc.PHI(j);
                    }
                }
                R s, mb, w;
                pair_props<R, SINGLE>(a, idk, idm, T, s, mb, w);
                cm -= s * pair_a<R, SINGLE>(sc, k, w);
                if (pk != (R)0) {
                    for (int q = q0; q < nz; q++) {     /* i > m */
                        const int i = sc.NZ(q);
                        if (i <= m) continue;
                        const R t = triple_weight<R, SINGLE>(a, idk, idm, sc.ID(i), T);
                        cm -= t * pk * sc.PHI(i);
                    }
                }
            }
            int q1 = 0;
            for (int j = m + 1; j < n; j++) {
                R s, mb, w;
                const int idj = sc.ID(j);
                pair_props<R, SINGLE>(a, idm, idj, T, s, mb, w);
                cm -= s * pair_a<R, SINGLE>(sc, j, w);
                const R pj = sc.PHI(j);
                if (pj != (R)0) {
                    while (q1 < nz && sc.NZ(q1) <= j) q1++;
                    for (int q = q1; q < nz; q++) {     /* i > j */
                        const int i = sc.NZ(q);
                        const R t = triple_weight<R, SINGLE>(a, idm, idj, sc.ID(i), T);
                        cm -= t * pj * sc.PHI(i);
                    }
                }
            }
            cm *= (R)8.0;
            cm += sc.LAP(m);
            sc.CAP(m) = cm;
        }
        /* unconstrained rate and active set (src/cipher.c:524-539) */
        for (int m = 0; m < n; m++) {
            R u = (R)0;
            const R cmv = sc.CAP(m);
            const int idm = sc.ID(m);
            for (int k = 0; k < m; k++) {
                R s, mb, w;
                pair_props<R, SINGLE>(a, sc.ID(k), idm, T, s, mb, w);
                u -= mb * (sc.CAP(k) - cmv);
            }
            for (int j = m + 1; j < n; j++) {
                R s, mb, w;
                pair_props<R, SINGLE>(a, idm, sc.ID(j), T, s, mb, w);
                u += mb * (cmv - sc.CAP(j));
            }
            const double p = (double)sc.PHI(m);
            const bool on = (p > CIPHER_TOL && p < 1.0 - CIPHER_TOL) || (p < CIPHER_TOL && u > (R)0) ||
                            (p > 1.0 - CIPHER_TOL && u < (R)0);
            if (on) { act |= 1u << m; nact += (R)1.0; }
        }
    }
    if (!live) return;
    /* constrained rate (src/cipher.c:541-555), written for all P slots */
    for (int m = 0; m < a.P; m++) {
        R v = (R)0;
        if (m < n && (act >> m & 1u)) {
            const R cmv = sc.CAP(m);
            const int idm = sc.ID(m);
            for (int k = 0; k < m; k++) {
                if (!(act >> k & 1u)) continue;
                R s, mb, w;
                pair_props<R, SINGLE>(a, sc.ID(k), idm, T, s, mb, w);
                v -= mb * (sc.CAP(k) - cmv);
            }
            for (int j = m + 1; j < n; j++) {
                if (!(act >> j & 1u)) continue;
                R s, mb, w;
                pair_props<R, SINGLE>(a, idm, sc.ID(j), T, s, mb, w);
                v += mb * (cmv - sc.CAP(j));
            }
            v /= nact;
        }
        a.fphi[(int64_t)m * S + c] = v;
    }
}

}  // namespace cipher
