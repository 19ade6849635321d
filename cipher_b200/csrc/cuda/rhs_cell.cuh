/*
 * rhs_cell.cuh - per-cell face gather for the phase-field RHS on uniform
 * grids (the face loop of src/cipher.c:235-317 turned into a gather).
 *
 * One thread per cell, launch grid (x-blocks, y, z).  The cell's own slots
 * (ids, phase fractions, Laplacian) live in registers: every loop over them is
 * unrolled to the compile-time slot bound PM with a warp-uniform early exit,
 * so their indices are constants.  Each neighbour's set is first copied into
 * a small per-thread shared-memory scratch with independent loads (one
 * memory latency per face), then merged against the own set: the own side
 * advances by the unrolled slot index, the neighbour side by a data-dependent
 * pointer into the scratch.
 *
 * Face order: the reference adds face fluxes in face order, faces being
 * (c, c+e_d) by ascending c then d.  For a cell that is: faces whose L cell
 * lies below without wrap (descending d), its own faces (ascending d), then
 * the periodic faces whose L cell wraps around from above (ascending d).
 */
#pragma once
#include <cstdint>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"

namespace cipher {

template <int PM, typename R>
struct OwnSlots {
    uint16_t ids[PM];
    R phi[PM];
    R lap[PM];
    int n;
};

/* per-thread neighbour scratch in shared memory: ids [PM][bd], phi [PM][bd] */
template <typename R>
struct NbScratch {
    uint16_t *ids;
    R *phi;
    int st;
};

/* neighbour at fixed face position f of a cell: [0,DIM) below without wrap
 * (descending d), [DIM,2DIM) own faces (ascending d), [2DIM,3DIM) wrapped
 * from above (ascending d); -1 if the face is absent.  Cell indices fit in
 * 31 bits (checked when the context is created). */
template <int DIM>
__device__ __forceinline__ int face_nb(const int *res, const int *per, int c, int x, int y, int z, int f)
{
    const int co[3] = {x, y, z};
    const int st[3] = {1, res[0], res[0] * res[1]};
    if (f < DIM) {
        const int e = DIM - 1 - f;
        return co[e] > 0 ? c - st[e] : -1;
    }
    if (f < 2 * DIM) {
        const int d = f - DIM;
        if (co[d] < res[d] - 1) return c + st[d];
        return (per[d] && res[d] > 1) ? c - (res[d] - 1) * st[d] : -1;
    }
    const int d = f - 2 * DIM;
    return (co[d] == 0 && per[d] && res[d] > 1) ? c + (res[d] - 1) * st[d] : -1;
}

template <int PM, typename R, bool EXACT>
__device__ __forceinline__ void cell_face(const PfArgs<R> &a, OwnSlots<PM, R> &o, int nw, int nb, int nn,
                                          bool cell_is_L, const NbScratch<R> &sc)
{
    const int64_t S = a.stride;
    if (nn > a.P) nn = a.P;                 /* that cell's own thread raises the flag */
    if (nn < 1 || o.n < 1) return;
    /* independent loads of the neighbour's set into the scratch */
    for (int j = 0; j < nn; j++) {
        sc.ids[j * sc.st] = __ldg(&a.as[(int64_t)(1 + j) * S + nb]);
        sc.phi[j * sc.st] = __ldg(&a.phi[(int64_t)j * S + nb]);
    }
    const uint16_t b0 = sc.ids[0];
    /* the phase flux is gated on the L cell only (src/cipher.c:277) */
    const bool gate = cell_is_L ? (o.n > 1 || o.ids[0] > 1) : (nn > 1 || b0 > 1);
    if (!gate) return;
    int j = 0;
    uint16_t b = b0;
#pragma unroll
    for (int g = 0; g < PM; g++) {
        if (g >= nw) break;                 /* warp-uniform */
        if (g < o.n) {
            const uint16_t v = o.ids[g];
            while (b < v) {
                if (++j >= nn) { b = 0xFFFF; break; }
                b = sc.ids[j * sc.st];
            }
            if (b == v) {
                const R pn = sc.phi[j * sc.st];
                if (cell_is_L) o.lap[g] += face_term<R, EXACT>(a, pn - o.phi[g]);
                else o.lap[g] -= face_term<R, EXACT>(a, o.phi[g] - pn);
                b = ++j < nn ? sc.ids[j * sc.st] : 0xFFFF;
            }
        }
    }
}

/* load the own set (flag invalid cells; n = 0 for them and dead threads),
 * then gather all faces in the reference's order.  Returns the warp-max n. */
template <int DIM, int PM, typename R, bool EXACT>
__device__ __forceinline__ int cell_gather(const PfArgs<R> &a, int c, bool live, int x, int y, int z,
                                           OwnSlots<PM, R> &o, const NbScratch<R> &sc)
{
    const int64_t S = a.stride;
    int n = live ? (int)__ldg(&a.as[c]) : 0;
    /* every neighbour's count, packed 4 bits per face (counts above P are
     * clamped to P; their own threads raise the flag) */
    uint64_t nnp = 0;
#pragma unroll
    for (int f = 0; f < 3 * DIM; f++) {
        const int nb = live ? face_nb<DIM>(a.res, a.per, c, x, y, z, f) : -1;
        int k = nb >= 0 ? (int)__ldg(&a.as[nb]) : 0;
        k = k > a.P ? a.P : k;
        nnp |= (uint64_t)k << (4 * f);
    }
    bool ok = true;
    if (live && (n < 1 || n > a.P)) { ok = false; n = 0; }
#pragma unroll
    for (int g = 0; g < PM; g++) {
        o.lap[g] = (R)0;
        if (g < n) {
            o.ids[g] = __ldg(&a.as[(int64_t)(1 + g) * S + c]);
            o.phi[g] = __ldg(&a.phi[(int64_t)g * S + c]);
            ok = ok && o.ids[g] < a.npf;
        } else {
            o.ids[g] = 0xFFFF;
            o.phi[g] = (R)0;
        }
    }
    if (!ok) {
        atomicOr(a.err, ERR_BADSET);
        n = 0;
    }
    o.n = n;
    const int nw = __reduce_max_sync(0xffffffffu, (unsigned)n);
    if (n > 0) {
#pragma unroll
        for (int f = 0; f < 3 * DIM; f++) {
            const int nb = face_nb<DIM>(a.res, a.per, c, x, y, z, f);
            if (nb >= 0) cell_face<PM, R, EXACT>(a, o, nw, nb, (int)(nnp >> (4 * f) & 15u), f >= DIM && f < 2 * DIM, sc);
        }
    }
    return nw;
}

}  // namespace cipher
