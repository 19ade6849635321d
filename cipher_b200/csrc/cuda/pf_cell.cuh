/*
 * pf_cell.cuh - cell terms of the phase-field RHS in the reference's
 * operation order (src/cipher.c:417-555): capillary force with the
 * triple-junction penalty, the unconstrained pair rates, the active set and
 * the constrained rate.
 *
 * The reference accumulates each slot's capillary force inside a k<j<i loop
 * nest that also updates the other slots.  Each slot m receives, in order:
 *   for k < m:  -t(k,j,m) phi_k phi_j   for k < j < m   (m as the third phase)
 *               -sigma(k,m) a_k(k,m)                     (m as the second)
 *               -t(k,m,i) phi_k phi_i   for i > m        (m as the second)
 *   then        -sigma(m,j) a_j(m,j), -t(m,j,i) phi_j phi_i  for j > m, i > j
 *   then        *8, + lap_m
 * with a_j(k,m) = phi_j/w + lap_j*w/pi/pi.  Evaluating that sequence per
 * slot gives the same IEEE results while each slot's chain is independent.
 * The rates follow the same per-slot decomposition.  The cell's slots are
 * staged in shared memory (one column per thread) so the loops index them
 * freely without local-memory traffic.
 */
#pragma once
#include <cstdint>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"

namespace cipher {

template <typename R>
struct SlotColumns {
    R *phi, *aj, *lap, *cap;
    uint16_t *ids;
    int st;                      /* distance between slots of one thread */
    __device__ R &PHI(int g) const { return phi[g * st]; }
    __device__ R &AJ(int g) const { return aj[g * st]; }
    __device__ R &LAP(int g) const { return lap[g * st]; }
    __device__ R &CAP(int g) const { return cap[g * st]; }
    __device__ uint16_t &ID(int g) const { return ids[g * st]; }
};

/* pair sigma, m, w of phases (ids) a<b at temperature T */
template <typename R>
__device__ __forceinline__ void pair_props(const PfArgs<R> &a, int ia, int ib, double T, R &sig, R &mob, R &wid)
{
    if (a.single) {
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
template <typename R>
__device__ __forceinline__ R triple_weight(const PfArgs<R> &a, int ia, int ib, int ic, double T)
{
    if (a.single) return (R)a.tj0;
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

/* capillary term of phase j as seen by the pair (p, q) it belongs to */
template <typename R>
__device__ __forceinline__ R pair_a(const SlotColumns<R> &sc, int j, R wid)
{
    const R PI = (R)CIPHER_PI_D;
    return sc.PHI(j) / wid + sc.LAP(j) * wid / PI / PI;
}

/*
 * Cell terms in reference order; writes all P slots of F for this cell.
 * n: active count (0 for dead/invalid threads, which write nothing when !live).
 */
template <int PM, typename R>
__device__ __forceinline__ void cell_rates_ordered(const PfArgs<R> &a, const CellPF<PM, R> &cp,
                                                   const SlotColumns<R> &sc, int64_t c, bool live, double T)
{
    const int n = cp.n;
    const int64_t S = a.stride;
#pragma unroll
    for (int g = 0; g < PM; g++) {
        if (g < n) {
            sc.PHI(g) = cp.phi[g];
            sc.LAP(g) = cp.lap[g];
            sc.ID(g) = cp.ids[g];
        }
    }
    const bool single = a.single;
    R sig1 = 0, mob1 = 0, wid1 = 0;
    if (single && n > 1) {
        /* with one interface a_j does not depend on the pair: form it once */
        pair_props<R>(a, 0, 0, T, sig1, mob1, wid1);
        for (int g = 0; g < n; g++) sc.AJ(g) = pair_a<R>(sc, g, wid1);
    }
    if (n > 1) {
        /* capillary force per slot */
        for (int m = 0; m < n; m++) {
            R cm = (R)0;
            const int idm = sc.ID(m);
            for (int k = 0; k < m; k++) {
                const R pk = sc.PHI(k);
                const int idk = sc.ID(k);
                for (int j = k + 1; j < m; j++) {
                    R t = triple_weight<R>(a, idk, sc.ID(j), idm, T);
                    cm -= t * pk * sc.PHI(j);
                }
                R s, mb, w;
                pair_props<R>(a, idk, idm, T, s, mb, w);
                cm -= s * (single ? sc.AJ(k) : pair_a<R>(sc, k, w));
                for (int i = m + 1; i < n; i++) {
                    R t = triple_weight<R>(a, idk, idm, sc.ID(i), T);
                    cm -= t * pk * sc.PHI(i);
                }
            }
            for (int j = m + 1; j < n; j++) {
                R s, mb, w;
                const int idj = sc.ID(j);
                pair_props<R>(a, idm, idj, T, s, mb, w);
                cm -= s * (single ? sc.AJ(j) : pair_a<R>(sc, j, w));
                const R pj = sc.PHI(j);
                for (int i = j + 1; i < n; i++) {
                    R t = triple_weight<R>(a, idm, idj, sc.ID(i), T);
                    cm -= t * pj * sc.PHI(i);
                }
            }
            cm *= (R)8.0;
            cm += sc.LAP(m);
            sc.CAP(m) = cm;
        }
    }
    /* unconstrained rate and active set (src/cipher.c:524-539) */
    uint32_t act = 0;
    R nact = (R)0;
    if (n > 1) {
        for (int m = 0; m < n; m++) {
            R u = (R)0;
            const R cmv = sc.CAP(m);
            const int idm = sc.ID(m);
            for (int k = 0; k < m; k++) {
                R s, mb, w;
                pair_props<R>(a, sc.ID(k), idm, T, s, mb, w);
                u -= mb * (sc.CAP(k) - cmv);
            }
            for (int j = m + 1; j < n; j++) {
                R s, mb, w;
                pair_props<R>(a, idm, sc.ID(j), T, s, mb, w);
                u += mb * (cmv - sc.CAP(j));
            }
            const double p = (double)sc.PHI(m);
            const bool on = (p > CIPHER_TOL && p < 1.0 - CIPHER_TOL) || (p < CIPHER_TOL && u > (R)0) ||
                            (p > 1.0 - CIPHER_TOL && u < (R)0);
            if (on) { act |= 1u << m; nact += (R)1.0; }
        }
    }
    /* constrained rate (src/cipher.c:541-555), written for all P slots */
    for (int m = 0; m < a.P; m++) {
        R v = (R)0;
        if (m < n && (act >> m & 1u)) {
            const R cmv = sc.CAP(m);
            const int idm = sc.ID(m);
            for (int k = 0; k < m; k++) {
                if (!(act >> k & 1u)) continue;
                R s, mb, w;
                pair_props<R>(a, sc.ID(k), idm, T, s, mb, w);
                v -= mb * (sc.CAP(k) - cmv);
            }
            for (int j = m + 1; j < n; j++) {
                if (!(act >> j & 1u)) continue;
                R s, mb, w;
                pair_props<R>(a, idm, sc.ID(j), T, s, mb, w);
                v += mb * (cmv - sc.CAP(j));
            }
            v /= nact;
        }
        if (live) a.fphi[(int64_t)m * S + c] = v;
    }
}

}  // namespace cipher
