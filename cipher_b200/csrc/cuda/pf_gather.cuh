/*
 * pf_gather.cuh - per-cell phase-field Laplacian gathered over the faces of a
 * uniform grid, for the phase-field RHS kernels.
 *
 * The reference scatters each face's flux into both cells (src/cipher.c:
 * 235-317); here every cell gathers the contributions of its own faces, in
 * the order the reference's face loop reaches them, so each slot receives
 * the same additions in the same order.  The cell's slots live in shared
 * memory, one column per thread (SlotColumns).  Which neighbour slot holds
 * each own phase (SetIntersection, src/utility.c:168-190, with the gate of
 * src/cipher.c:277) is read from the state's face maps, built from the sets
 * when they change (poststep.cu: build_maps_row), so the RHS does no set
 * merging at all.
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

/* a thread's slot columns in shared memory, one entry per slot g at
 * base[g*st] */
template <typename R>
struct SlotColumns {
    R *phi, *aj, *lap, *cap;
    uint16_t *ids;
    uint8_t *nz;                 /* slots with phi != 0, ascending */
    int st;
    __device__ __forceinline__ R &PHI(int g) const { return phi[g * st]; }
    __device__ __forceinline__ R &AJ(int g) const { return aj[g * st]; }
    __device__ __forceinline__ R &LAP(int g) const { return lap[g * st]; }
    __device__ __forceinline__ R &CAP(int g) const { return cap[g * st]; }
    __device__ __forceinline__ uint16_t &ID(int g) const { return ids[g * st]; }
    __device__ __forceinline__ uint8_t &NZ(int g) const { return nz[g * st]; }
};

/* carve the columns of thread `tid` out of a block's dynamic shared memory;
 * layout: R phi,lap[,aj,cap] [PM][bd] | uint16 ids [PM][bd] | uint8 nz [PM][bd] */
template <typename R>
__device__ __forceinline__ SlotColumns<R> slot_columns(unsigned char *smem, int PM, int bd, int tid, bool with_aj_cap)
{
    SlotColumns<R> sc;
    R *base = (R *)smem;
    int k = 0;
    sc.st = bd;
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

/* cell index and coordinates of this thread */
struct CellIndex {
    int64_t c;
    int x, y, z;
    bool live;
};

/* blocks of BX x BY cells in (x, y); grid (ceil(res0/BX), ceil(res1/BY),
 * planes), plane zbase + blockIdx.z */
template <int BX, int BY>
__device__ __forceinline__ CellIndex cell_index(const int *res, int zbase = 0)
{
    CellIndex ci;
    ci.x = blockIdx.x * BX + (int)threadIdx.x % BX;
    ci.y = blockIdx.y * BY + (int)threadIdx.x / BX;
    ci.z = zbase + (int)blockIdx.z;
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

/* face-map direction of face position f: 2d for the lower neighbour along
 * d (without or with wrap), 2d+1 for the upper one */
template <int DIM>
__device__ __forceinline__ int face_dir(int f)
{
    if (f < DIM) return 2 * (DIM - 1 - f);
    if (f < 2 * DIM) return 2 * (f - DIM) + 1;
    return 2 * (f - 2 * DIM);
}

/* load the cell's phase fractions (and ids when IDS) into its columns and
 * gather its faces in the reference's face order through the face maps.
 * Returns the active count (0 for a dead or invalid cell; an invalid count
 * raises ERR_BADSET). */
template <int DIM, int PM, typename R, bool EXACT, bool IDS>
__device__ __forceinline__ int load_and_gather(const PfArgs<R> &a, const CellIndex &ci, const SlotColumns<R> &sc)
{
    const int64_t S = a.stride, c = ci.c;
    int n = ci.live ? (int)__ldg(&a.as[c]) : 0;
    if (ci.live && (n < 1 || n > a.P)) {
        atomicOr(a.err, ERR_BADSET);
        return 0;
    }
    if (n == 0) return 0;
    int64_t nbs[3 * DIM];
#pragma unroll
    for (int f = 0; f < 3 * DIM; f++) nbs[f] = face_nb<DIM, R>(a, ci, f);
    for (int g0 = 0; g0 < n; g0 += 4) {
        R tp[4];
        uint16_t ti[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (g0 + k < n) {
                tp[k] = __ldg(&a.phi[(int64_t)(g0 + k) * S + c]);
                if (IDS) ti[k] = __ldg(&a.as[(int64_t)(1 + g0 + k) * S + c]);
            }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (g0 + k < n) {
                sc.PHI(g0 + k) = tp[k];
                sc.LAP(g0 + k) = (R)0;
                if (IDS) sc.ID(g0 + k) = ti[k];
            }
        }
    }
    /* four slots at a time: their face-map words, then for each face in the
     * reference's order the matched neighbour slots (loads issue together).
     * Each slot still receives its faces' contributions in face order. */
    for (int i0 = 0; i0 < n; i0 += 4) {
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; k++) w[k] = i0 + k < n ? __ldg(&a.maps[(int64_t)(i0 + k) * S + c]) : ~0u;
#pragma unroll
        for (int f = 0; f < 3 * DIM; f++) {
            const int64_t nb = nbs[f];
            if (nb < 0) continue;
            const bool cell_is_L = f >= DIM && f < 2 * DIM;
            const unsigned sh = 4u * (unsigned)face_dir<DIM>(f);
            R pn[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int j = (int)((w[k] >> sh) & 15u);
                pn[k] = (i0 + k < n && j < a.P) ? __ldg(&a.phi[(int64_t)j * S + nb]) : (R)0;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int i = i0 + k;
                const int j = (int)((w[k] >> sh) & 15u);
                if (i < n && j < a.P) {
                    if (cell_is_L) sc.LAP(i) += face_term<R, EXACT>(a, pn[k] - sc.PHI(i));
                    else sc.LAP(i) -= face_term<R, EXACT>(a, sc.PHI(i) - pn[k]);
                }
            }
        }
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
