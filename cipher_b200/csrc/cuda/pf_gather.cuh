/*
 * pf_gather.cuh - per-cell phase-field Laplacian gathered over the faces of a
 * uniform grid, for the phase-field RHS kernels.
 *
 * The reference scatters each face's flux into both cells (src/cipher.c:
 * 235-317); here every cell gathers the contributions of its own faces, in
 * the order the reference's face loop reaches them, so each slot receives
 * the same additions in the same order.  Slot arrays stay in registers: the
 * own set is held in fixed-size arrays indexed only by unrolled constants,
 * and a neighbour's phase is matched against all own slots by comparison
 * instead of a merge with data-dependent indices.
 */
#pragma once
#include <cstdint>
#include "device_common.cuh"
#include "kernels.h"

namespace cipher {

/* how a face contribution ff*flux/vol is formed */
enum GeomMode : int {
    GEOM_DIVIDE = 0,    /* (ff*flux)/vol, as the reference writes it */
    GEOM_RECIP = 1,     /* vol a power of two: (ff*flux)*(1/vol), exact */
    GEOM_UNIT = 2,      /* ff == 1 and vol == 1: flux itself, exact */
};

template <int PM, typename R>
struct CellPF {
    uint16_t ids[PM];
    R phi[PM];
    R lap[PM];
    int n;
    uint16_t maxid;
};

template <typename R, bool EXACT>
__device__ __forceinline__ R face_term(const PfArgs<R> &a, R flux)
{
    if (EXACT) {
        if (a.geom_mode == GEOM_UNIT) return flux;
        if (a.geom_mode == GEOM_RECIP) return ((R)a.ffactor * flux) * (R)a.inv_vol;
        return ((R)a.ffactor * flux) / (R)a.vol;
    } else {
        return (R)a.face_coef * flux;
    }
}

/* contributions of the face shared with neighbour nb (src/cipher.c:277-288) */
template <int PM, typename R, bool EXACT>
__device__ __forceinline__ void gather_face(const PfArgs<R> &a, CellPF<PM, R> &cp, int64_t nb, bool cell_is_L)
{
    const int64_t S = a.stride;
    int nn = a.as[nb];
    if (nn > a.P) nn = a.P;                 /* that cell's own thread raises the flag */
    if (nn < 1 || cp.n < 1) return;
    uint16_t b0 = a.as[S + nb];
    /* the phase flux is gated on the L cell only (src/cipher.c:277) */
    bool gate = cell_is_L ? (cp.n > 1 || cp.ids[0] > 1) : (nn > 1 || b0 > 1);
    if (!gate) return;
    for (int j = 0; j < nn; j++) {
        uint16_t nid = j == 0 ? b0 : a.as[(int64_t)(1 + j) * S + nb];
        if (nid > cp.maxid) break;          /* both sets are sorted */
        int mi = -1;
#pragma unroll
        for (int i = 0; i < PM; i++)
            if (i < cp.n && cp.ids[i] == nid) mi = i;
        if (mi < 0) continue;
        R pn = a.phi[(int64_t)j * S + nb];
#pragma unroll
        for (int i = 0; i < PM; i++) {
            if (i == mi) {
                if (cell_is_L) cp.lap[i] += face_term<R, EXACT>(a, pn - cp.phi[i]);
                else cp.lap[i] -= face_term<R, EXACT>(a, cp.phi[i] - pn);
            }
        }
    }
}

/* load the cell's set and phase fractions, then gather its faces in the
 * reference's face order (non-wrapped faces from below in descending
 * direction, own faces in ascending direction, wrapped faces from above in
 * ascending direction).  Returns false for an invalid cell (flag raised). */
template <int DIM, int PM, typename R, bool EXACT>
__device__ __forceinline__ bool load_and_gather(const PfArgs<R> &a, int64_t c, bool live, CellPF<PM, R> &cp)
{
    const int64_t S = a.stride;
    int n = live ? (int)a.as[c] : 0;
    bool ok = true;
    if (live && (n < 1 || n > a.P)) { ok = false; n = 0; }
    uint16_t maxid = 0;
#pragma unroll
    for (int g = 0; g < PM; g++) {
        if (g < n) {
            cp.ids[g] = a.as[(int64_t)(1 + g) * S + c];
            cp.phi[g] = a.phi[(int64_t)g * S + c];
            if (cp.ids[g] >= a.npf) ok = false;
            maxid = cp.ids[g];
        } else {
            cp.ids[g] = 0xFFFF;
            cp.phi[g] = (R)0;
        }
        cp.lap[g] = (R)0;
    }
    if (!ok) {
        atomicOr(a.err, ERR_BADSET);
        n = 0;
    }
    cp.n = n;
    cp.maxid = maxid;
    if (n == 0) return ok;

    const int res0 = a.res[0], res1 = a.res[1], res2 = a.res[2];
    const int64_t st1 = res0, st2 = (int64_t)res0 * res1;
    int co0 = (int)(c % res0);
    int co1 = DIM > 1 ? (int)((c / res0) % res1) : 0;
    int co2 = DIM > 2 ? (int)(c / st2) : 0;
    /* faces whose L cell lies below without wrapping, descending direction */
    if (DIM > 2 && co2 > 0) gather_face<PM, R, EXACT>(a, cp, c - st2, false);
    if (DIM > 1 && co1 > 0) gather_face<PM, R, EXACT>(a, cp, c - st1, false);
    if (co0 > 0) gather_face<PM, R, EXACT>(a, cp, c - 1, false);
    /* own faces, ascending direction */
    if (co0 < res0 - 1) gather_face<PM, R, EXACT>(a, cp, c + 1, true);
    else if (a.per[0]) gather_face<PM, R, EXACT>(a, cp, c - (res0 - 1), true);
    if (DIM > 1) {
        if (co1 < res1 - 1) gather_face<PM, R, EXACT>(a, cp, c + st1, true);
        else if (a.per[1]) gather_face<PM, R, EXACT>(a, cp, c - (int64_t)(res1 - 1) * st1, true);
    }
    if (DIM > 2) {
        if (co2 < res2 - 1) gather_face<PM, R, EXACT>(a, cp, c + st2, true);
        else if (a.per[2]) gather_face<PM, R, EXACT>(a, cp, c - (int64_t)(res2 - 1) * st2, true);
    }
    /* faces whose L cell wraps around from above, ascending direction */
    if (co0 == 0 && a.per[0]) gather_face<PM, R, EXACT>(a, cp, c + (res0 - 1), false);
    if (DIM > 1 && co1 == 0 && a.per[1]) gather_face<PM, R, EXACT>(a, cp, c + (int64_t)(res1 - 1) * st1, false);
    if (DIM > 2 && co2 == 0 && a.per[2]) gather_face<PM, R, EXACT>(a, cp, c + (int64_t)(res2 - 1) * st2, false);
    return ok;
}

}  // namespace cipher
