/*
 * pf_gather.cuh - per-cell phase-field Laplacian gathered over the faces of a
 * uniform grid, for the phase-field RHS kernels.
 *
 * The reference scatters each face's flux into both cells (src/cipher.c:
 * 235-317); here every cell gathers the contributions of its own faces, in
 * the order the reference's face loop reaches them, so each slot receives
 * the same additions in the same order.  The cell's slots live in shared
 * memory, one column per thread (SlotColumns), and a face is matched by a
 * two-pointer merge of the two sorted sets, as SetIntersection does
 * (src/utility.c:168-190).
 *
 * Launch geometry: grid (ceil(res0/block), res1, res2), one thread per cell
 * of an x-row, so cell coordinates need no integer division.
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

/* a thread's slot columns in shared memory: phi and ids at base[g*pst]
 * (a staged tile plane or a private column), the rest at base[g*st] */
template <typename R>
struct SlotColumns {
    R *phi, *aj, *lap, *cap;
    uint16_t *ids;
    uint8_t *nz;                 /* slots with phi != 0, ascending */
    int st, pst;
    __device__ __forceinline__ R &PHI(int g) const { return phi[g * pst]; }
    __device__ __forceinline__ R &AJ(int g) const { return aj[g * st]; }
    __device__ __forceinline__ R &LAP(int g) const { return lap[g * st]; }
    __device__ __forceinline__ R &CAP(int g) const { return cap[g * st]; }
    __device__ __forceinline__ uint16_t &ID(int g) const { return ids[g * pst]; }
    __device__ __forceinline__ uint8_t &NZ(int g) const { return nz[g * st]; }
};

/* carve the columns of thread `tid` out of a block's dynamic shared memory;
 * layout: R phi,aj,lap,cap [PM][bd] | uint16 ids [PM][bd] | uint8 nz [PM][bd] */
template <typename R>
__device__ __forceinline__ SlotColumns<R> slot_columns(unsigned char *smem, int PM, int bd, int tid, bool with_aj_cap)
{
    SlotColumns<R> sc;
    R *base = (R *)smem;
    int k = 0;
    sc.st = bd;
    sc.pst = bd;
    sc.phi = base + (size_t)(k++) * PM * bd + tid;
    sc.lap = base + (size_t)(k++) * PM * bd + tid;
    if (with_aj_cap) {
        sc.aj = base + (size_t)(k++) * PM * bd + tid;
        sc.cap = base + (size_t)(k++) * PM * bd + tid;
    } else {
        sc.aj = sc.cap = nullptr;
    }
    uint16_t *ib = (uint16_t *)(base + (size_t)k * PM * bd);
    sc.ids = ib + tid;
    sc.nz = (uint8_t *)(ib + (size_t)PM * bd) + tid;
    return sc;
}

__host__ __device__ constexpr size_t slot_columns_bytes(int PM, int bd, int rbytes, bool with_aj_cap)
{
    return (size_t)PM * bd * ((with_aj_cap ? 4 : 2) * rbytes + 2 + 1) + 16;
}

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

/* contributions of the face shared with neighbour nb whose active count nn
 * was already loaded (src/cipher.c:277-288).  The neighbour's ids and phase
 * fractions are loaded up front (independent loads, registers), then merged
 * against the cell's own sorted set in its columns. */
template <int PM, typename R, bool EXACT>
__device__ __forceinline__ void gather_face(const PfArgs<R> &a, const SlotColumns<R> &sc, int n, int64_t nb, int nn,
                                            bool cell_is_L)
{
    const int64_t S = a.stride;
    if (nn > a.P) nn = a.P;                 /* that cell's own thread raises the flag */
    if (nn < 1) return;
    uint16_t nid[PM];
    R nph[PM];
#pragma unroll
    for (int j = 0; j < PM; j++) {
        if (j < nn) {
            nid[j] = a.as[(int64_t)(1 + j) * S + nb];
            nph[j] = a.phi[(int64_t)j * S + nb];
        }
    }
    /* the phase flux is gated on the L cell only (src/cipher.c:277) */
    const bool gate = cell_is_L ? (n > 1 || sc.ID(0) > 1) : (nn > 1 || nid[0] > 1);
    if (!gate) return;
    int i = 0;
    uint16_t v = sc.ID(0);
#pragma unroll
    for (int j = 0; j < PM; j++) {
        if (j >= nn) break;
        const uint16_t b = nid[j];
        while (v < b) {
            if (++i >= n) return;
            v = sc.ID(i);
        }
        if (v == b) {
            if (cell_is_L) sc.LAP(i) += face_term<R, EXACT>(a, nph[j] - sc.PHI(i));
            else sc.LAP(i) -= face_term<R, EXACT>(a, sc.PHI(i) - nph[j]);
            if (++i >= n) return;
            v = sc.ID(i);
        }
    }
}

/* cell index and coordinates of this thread */
struct CellIndex {
    int64_t c;
    int x, y, z;
    bool live;
};

__device__ __forceinline__ CellIndex cell_index(const int *res)
{
    CellIndex ci;
    ci.x = blockIdx.x * blockDim.x + threadIdx.x;
    ci.y = blockIdx.y;
    ci.z = blockIdx.z;
    ci.live = ci.x < res[0];
    ci.c = (int64_t)ci.x + (int64_t)res[0] * ((int64_t)ci.y + (int64_t)res[1] * ci.z);
    return ci;
}

/* load the cell's set and phase fractions into its columns, then gather its
 * faces in the reference's face order (non-wrapped faces from below in
 * descending direction, own faces in ascending direction, wrapped faces
 * from above in ascending direction).  Returns the active count (0 for a
 * dead or invalid cell; an invalid one raises ERR_BADSET). */
template <int DIM, int PM, typename R, bool EXACT>
__device__ __forceinline__ int load_and_gather(const PfArgs<R> &a, const CellIndex &ci, const SlotColumns<R> &sc)
{
    const int64_t S = a.stride, c = ci.c;
    const int res0 = a.res[0], res1 = a.res[1], res2 = a.res[2];
    const int64_t st1 = res0, st2 = (int64_t)res0 * res1;
    const int co0 = ci.x, co1 = ci.y, co2 = ci.z;
    /* the neighbours in the reference's face order, at fixed positions:
     * [0, DIM)       below without wrap, descending direction
     * [DIM, 2 DIM)   own faces (L = this cell), ascending direction
     * [2 DIM, 3 DIM) wrapped from above, ascending direction
     * -1 marks an absent face */
    const int co[3] = {co0, co1, co2};
    const int rs[3] = {res0, res1, res2};
    const int64_t st[3] = {1, st1, st2};
    int64_t nb[3 * DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const int e = DIM - 1 - d;                     /* descending direction */
        nb[d] = co[e] > 0 ? c - st[e] : -1;
        nb[DIM + d] = co[d] < rs[d] - 1 ? c + st[d] : (a.per[d] ? c - (int64_t)(rs[d] - 1) * st[d] : -1);
        nb[2 * DIM + d] = (co[d] == 0 && a.per[d]) ? c + (int64_t)(rs[d] - 1) * st[d] : -1;
    }

    /* own set and every neighbour's count: independent loads issued together */
    int n = ci.live ? (int)a.as[c] : 0;
    int nn[3 * DIM];
#pragma unroll
    for (int f = 0; f < 3 * DIM; f++) nn[f] = (ci.live && nb[f] >= 0) ? (int)a.as[nb[f]] : 0;
    bool ok = true;
    if (ci.live && (n < 1 || n > a.P)) { ok = false; n = 0; }
    for (int g = 0; g < n; g++) {
        uint16_t id = a.as[(int64_t)(1 + g) * S + c];
        sc.ID(g) = id;
        sc.PHI(g) = a.phi[(int64_t)g * S + c];
        sc.LAP(g) = (R)0;
        if (id >= a.npf) ok = false;
    }
    if (!ok) {
        atomicOr(a.err, ERR_BADSET);
        return 0;
    }
    if (n == 0) return 0;
#pragma unroll
    for (int f = 0; f < 3 * DIM; f++)
        if (nb[f] >= 0) gather_face<PM, R, EXACT>(a, sc, n, nb[f], nn[f], f >= DIM && f < 2 * DIM);
    return n;
}

/* number of phi != 0 slots recorded by load_and_gather */
template <typename R>
__device__ __forceinline__ int count_nonzero(const SlotColumns<R> &sc, int n)
{
    int nz = 0;
    for (int g = 0; g < n; g++) nz += sc.PHI(g) != (R)0;
    return nz;
}

}  // namespace cipher
