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
 * Launch geometry: blocks of BX x BY cells in (x, y), grid
 * (ceil(res0/BX), ceil(res1/BY), res2): cell coordinates need no integer
 * division by the grid size and a warp covers 32 consecutive x cells.
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
    R *nph;                      /* scratch: the neighbour being merged */
    uint16_t *nids;
    int st, pst;
    __device__ __forceinline__ R &PHI(int g) const { return phi[g * pst]; }
    __device__ __forceinline__ R &AJ(int g) const { return aj[g * st]; }
    __device__ __forceinline__ R &LAP(int g) const { return lap[g * st]; }
    __device__ __forceinline__ R &CAP(int g) const { return cap[g * st]; }
    __device__ __forceinline__ uint16_t &ID(int g) const { return ids[g * pst]; }
    __device__ __forceinline__ uint8_t &NZ(int g) const { return nz[g * st]; }
    __device__ __forceinline__ R &NPH(int g) const { return nph[g * st]; }
    __device__ __forceinline__ uint16_t &NID(int g) const { return nids[g * st]; }
};

/* carve the columns of thread `tid` out of a block's dynamic shared memory;
 * layout: R phi,lap,nph[,aj,cap] [PM][bd] | uint16 ids,nids [PM][bd] | uint8 nz [PM][bd] */
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
    sc.nph = base + (size_t)(k++) * PM * bd + tid;
    if (with_aj_cap) {
        sc.aj = base + (size_t)(k++) * PM * bd + tid;
        sc.cap = base + (size_t)(k++) * PM * bd + tid;
    } else {
        sc.aj = sc.cap = nullptr;
    }
    uint16_t *ib = (uint16_t *)(base + (size_t)k * PM * bd);
    sc.ids = ib + tid;
    sc.nids = ib + (size_t)PM * bd + tid;
    sc.nz = (uint8_t *)(ib + (size_t)2 * PM * bd) + tid;
    return sc;
}

__host__ __device__ constexpr size_t slot_columns_bytes(int PM, int bd, int rbytes, bool with_aj_cap)
{
    return (size_t)PM * bd * ((with_aj_cap ? 5 : 3) * rbytes + 2 * 2 + 1) + 16;
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
 * was already loaded (src/cipher.c:277-288).  Branch-free two-pointer merge
 * of the two sorted sets (SetIntersection, src/utility.c:168-190): both
 * pointers advance by predicate, so a warp's lanes stay converged; the
 * neighbour's entries are read through the read-only cache. */
template <int PM, typename R, bool EXACT>
__device__ __forceinline__ void gather_face(const PfArgs<R> &a, const SlotColumns<R> &sc, int n, int64_t nb, int nn,
                                            bool cell_is_L)
{
    const int64_t S = a.stride;
    if (nn < 1) return;
    /* the neighbour's set, staged in the scratch columns four slots at a
     * time: each group's loads issue back to back, so a face costs about
     * one memory latency per four slots instead of one per slot */
    for (int j0 = 0; j0 < nn; j0 += 4) {
        uint16_t ti[4];
        R tp[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (j0 + k < nn) {
                ti[k] = __ldg(a.as + (int64_t)(1 + j0 + k) * S + nb);
                tp[k] = __ldg(a.phi + (int64_t)(j0 + k) * S + nb);
            }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (j0 + k < nn) {
                sc.NID(j0 + k) = ti[k];
                sc.NPH(j0 + k) = tp[k];
            }
        }
    }
    uint16_t b = sc.NID(0);
    uint16_t v = sc.ID(0);
    /* the phase flux is gated on the L cell only (src/cipher.c:277) */
    const bool gate = cell_is_L ? (n > 1 || v > 1) : (nn > 1 || b > 1);
    if (!gate) return;
    int i = 0, j = 0;
    while (true) {
        if (v == b) {
            const R pn = sc.NPH(j);
            if (cell_is_L) sc.LAP(i) += face_term<R, EXACT>(a, pn - sc.PHI(i));
            else sc.LAP(i) -= face_term<R, EXACT>(a, sc.PHI(i) - pn);
        }
        i += v <= b;
        j += v >= b;
        if (i >= n || j >= nn) break;
        v = sc.ID(i);
        b = sc.NID(j);
    }
}

/* cell index and coordinates of this thread */
struct CellIndex {
    int64_t c;
    int x, y, z;
    bool live;
};

/* blocks of BX x BY cells in (x, y); grid (ceil(res0/BX), ceil(res1/BY), res2) */
template <int BX, int BY>
__device__ __forceinline__ CellIndex cell_index(const int *res)
{
    CellIndex ci;
    ci.x = blockIdx.x * BX + (int)threadIdx.x % BX;
    ci.y = blockIdx.y * BY + (int)threadIdx.x / BX;
    ci.z = blockIdx.z;
    ci.live = ci.x < res[0] && ci.y < res[1];
    ci.c = (int64_t)ci.x + (int64_t)res[0] * ((int64_t)ci.y + (int64_t)res[1] * ci.z);
    return ci;
}

/* cell of this thread in tile t of a batch; `inst` receives the domain.
 * Domains are found by binary search of the tile prefix (uniform across
 * the block, so no divergence). */
template <int BX, int BY, typename R>
__device__ __forceinline__ CellIndex batch_cell_index(const BatchTiles<R> &b, int64_t t, int &inst)
{
    int lo = 0, hi = b.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&b.tile_start[mid]) <= t) lo = mid;
        else hi = mid - 1;
    }
    inst = lo;
    const int *res = b.args[lo].res;
    const int r0 = res[0], r1 = res[1];
    const int64_t local = t - __ldg(&b.tile_start[lo]);
    const int tx = (r0 + BX - 1) / BX, ty = (r1 + BY - 1) / BY;
    const int bx = (int)(local % tx);
    const int by = (int)((local / tx) % ty);
    const int bz = (int)(local / ((int64_t)tx * ty));
    CellIndex ci;
    ci.x = bx * BX + (int)threadIdx.x % BX;
    ci.y = by * BY + (int)threadIdx.x / BX;
    ci.z = bz;
    ci.live = ci.x < r0 && ci.y < r1;
    ci.c = (int64_t)ci.x + (int64_t)r0 * ((int64_t)ci.y + (int64_t)r1 * ci.z);
    return ci;
}

/* neighbour at fixed face position f: [0,DIM) below without wrap
 * (descending d), [DIM,2DIM) own faces (ascending d), [2DIM,3DIM) wrapped
 * around from above (ascending d); -1 when the face is absent.  This is the
 * order in which the reference's face loop reaches the cell's faces. */
template <int DIM, typename R>
__device__ __forceinline__ int64_t face_nb(const PfArgs<R> &a, const CellIndex &ci, int f)
{
    const int co[3] = {ci.x, ci.y, ci.z};
    const int64_t st[3] = {1, (int64_t)a.res[0], (int64_t)a.res[0] * a.res[1]};
    if (f < DIM) {
        const int e = DIM - 1 - f;
        return co[e] > 0 ? ci.c - st[e] : -1;
    }
    if (f < 2 * DIM) {
        const int d = f - DIM;
        if (co[d] < a.res[d] - 1) return ci.c + st[d];
        return (a.per[d] && a.res[d] > 1) ? ci.c - (int64_t)(a.res[d] - 1) * st[d] : -1;
    }
    const int d = f - 2 * DIM;
    return (co[d] == 0 && a.per[d] && a.res[d] > 1) ? ci.c + (int64_t)(a.res[d] - 1) * st[d] : -1;
}

/* load the cell's set into its columns and gather its faces in the
 * reference's face order.  Returns the active count (0 for a dead or
 * invalid cell; an invalid one raises ERR_BADSET). */
template <int DIM, int PM, typename R, bool EXACT>
__device__ __forceinline__ int load_and_gather(const PfArgs<R> &a, const CellIndex &ci, const SlotColumns<R> &sc)
{
    const int64_t S = a.stride, c = ci.c;
    int n = ci.live ? (int)__ldg(&a.as[c]) : 0;
    /* the neighbours' counts, packed 4 bits per face position (clamped to P;
     * a neighbour's own thread flags an invalid count) */
    uint64_t nnp = 0;
#pragma unroll
    for (int f = 0; f < 3 * DIM; f++) {
        const int64_t nb = ci.live ? face_nb<DIM, R>(a, ci, f) : -1;
        int k = nb >= 0 ? (int)__ldg(&a.as[nb]) : 0;
        k = k > a.P ? a.P : k;
        nnp |= (uint64_t)k << (4 * f);
    }
    bool ok = true;
    if (ci.live && (n < 1 || n > a.P)) { ok = false; n = 0; }
    for (int g0 = 0; g0 < n; g0 += 4) {
        uint16_t ti[4];
        R tp[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (g0 + k < n) {
                ti[k] = __ldg(&a.as[(int64_t)(1 + g0 + k) * S + c]);
                tp[k] = __ldg(&a.phi[(int64_t)(g0 + k) * S + c]);
            }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (g0 + k < n) {
                sc.ID(g0 + k) = ti[k];
                sc.PHI(g0 + k) = tp[k];
                sc.LAP(g0 + k) = (R)0;
                if (ti[k] >= a.npf) ok = false;
            }
        }
    }
    if (!ok) {
        atomicOr(a.err, ERR_BADSET);
        return 0;
    }
    if (n == 0) return 0;
#pragma unroll
    for (int f = 0; f < 3 * DIM; f++) {
        const int nn = (int)(nnp >> (4 * f) & 15u);
        if (nn) gather_face<PM, R, EXACT>(a, sc, n, face_nb<DIM, R>(a, ci, f), nn, f >= DIM && f < 2 * DIM);
    }
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
