/*
 * rhs_tile.cuh - z-marching shared-memory tiles for the phase-field RHS on
 * uniform grids (the face loop of src/cipher.c:235-317 as a gather, and the
 * cell loop of src/cipher.c:391-555).
 *
 * A block owns a TX x TY column of cells in (x, y) and marches over ZC
 * z-planes.  Shared memory holds three z-planes (z-1, z, z+1) of the tile
 * plus a one-cell halo in x and y: per cell its active count, its P sorted
 * phase ids and its P phase fractions (only the n active slots are loaded).
 * Each new plane is fetched with independent, coalesced loads (a warp reads
 * 32 consecutive cells of one slot plane), so each cell's data crosses from
 * L2 about 1.6-2x per launch and from HBM once; every set merge of the face
 * gather then runs out of shared memory.
 *
 * Face order: the reference adds face fluxes in face order, faces being
 * (c, c+e_d) by ascending c then d.  For a cell that is: faces whose L cell
 * lies below without wrap (descending d), its own faces (ascending d), then
 * the periodic faces whose L cell wraps around from above (ascending d).
 * The gather follows it, so the FP64 instantiation is bit-identical.
 */
#pragma once
#include <cstdint>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"

namespace cipher {

template <int TX, int TY>
struct TileShape {
    static constexpr int HX = TX + 2;
    static constexpr int HY = TY + 2;
    static constexpr int HC = HX * HY;      /* halo cells per plane */
    static constexpr int NT = TX * TY;      /* threads per block */
};

/* one staged z-plane: phi [P][HC] | ids [P][HC] | cnt [HC] */
template <typename R>
struct TilePlane {
    R *phi;
    uint16_t *ids;
    uint8_t *cnt;
};

template <typename R, int HC>
__host__ __device__ constexpr size_t tile_plane_bytes(int P)
{
    return (((size_t)P * HC * (sizeof(R) + 2) + HC) + 15) / 16 * 16;
}

template <typename R, int HC>
__device__ __forceinline__ TilePlane<R> tile_plane(unsigned char *base, int P)
{
    TilePlane<R> pl;
    pl.phi = (R *)base;
    pl.ids = (uint16_t *)(pl.phi + (size_t)P * HC);
    pl.cnt = (uint8_t *)(pl.ids + (size_t)P * HC);
    return pl;
}

/* global index of halo cell (gx, gy, gz) with periodic wrap; -1 if absent */
template <int DIM>
__device__ __forceinline__ int64_t halo_cell(const int *res, const int *per, int gx, int gy, int gz)
{
    int g[3] = {gx, gy, gz};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int r = res[d];
        if (d >= DIM) {
            if (g[d] != 0) return -1;
            continue;
        }
        if (g[d] < 0 || g[d] >= r) {
            if (!per[d] || r < 2) return -1;
            g[d] = ((g[d] % r) + r) % r;
        }
    }
    return (int64_t)g[0] + (int64_t)res[0] * ((int64_t)g[1] + (int64_t)res[1] * g[2]);
}

/* stage plane gz of the tile at (x0, y0) (absent planes get count 0) */
template <int DIM, int TX, int TY, typename R>
__device__ __forceinline__ void load_tile_plane(const PfArgs<R> &a, const TilePlane<R> &pl, int x0, int y0, int gz,
                                                bool present)
{
    using T = TileShape<TX, TY>;
    const int64_t S = a.stride;
    for (int h = threadIdx.x; h < T::HC; h += T::NT) {
        const int hx = h % T::HX, hy = h / T::HX;
        /* corner halo cells are nobody's face neighbour */
        const bool corner = (hx == 0 || hx == T::HX - 1) && (hy == 0 || hy == T::HY - 1);
        int64_t c = -1;
        if (present && !corner) c = halo_cell<DIM>(a.res, a.per, x0 - 1 + hx, y0 - 1 + hy, gz);
        int n = c >= 0 ? (int)a.as[c] : 0;
        pl.cnt[h] = (uint8_t)(n > 255 ? 255 : n);
        if (n > a.P) n = a.P;
        for (int g = 0; g < n; g++) {
            pl.ids[g * T::HC + h] = a.as[(int64_t)(1 + g) * S + c];
            pl.phi[g * T::HC + h] = a.phi[(int64_t)g * S + c];
        }
    }
}

/* one face: neighbour at halo index hn of plane nbp (src/cipher.c:277-288) */
template <int HC, typename R, bool EXACT>
__device__ __forceinline__ void tile_face(const PfArgs<R> &a, const TilePlane<R> &own, int h0, int n,
                                          const TilePlane<R> &nbp, int hn, R *lap, int lst, bool cell_is_L)
{
    int nn = nbp.cnt[hn];
    if (nn > a.P) nn = a.P;
    if (nn < 1) return;
    uint16_t b = nbp.ids[hn];
    uint16_t v = own.ids[h0];
    /* the phase flux is gated on the L cell only (src/cipher.c:277) */
    const bool gate = cell_is_L ? (n > 1 || v > 1) : (nn > 1 || b > 1);
    if (!gate) return;
    /* branch-free two-pointer merge: both pointers advance by predicate, so
     * the lanes of a warp stay converged whatever their sets look like */
    const uint16_t *oi = own.ids + h0, *ni = nbp.ids + hn;
    const R *op = own.phi + h0, *np = nbp.phi + hn;
    int i = 0, j = 0;
    while (true) {
        if (v == b) {
            const R pn = np[j * HC], po = op[i * HC];
            if (cell_is_L) lap[i * lst] += face_term<R, EXACT>(a, pn - po);
            else lap[i * lst] -= face_term<R, EXACT>(a, po - pn);
        }
        i += v <= b;
        j += v >= b;
        if (i >= n || j >= nn) break;
        v = oi[i * HC];
        b = ni[j * HC];
    }
}

/* gather all faces of the cell at (gx,gy,gz), tile position (tx,ty) */
template <int DIM, int TX, int TY, typename R, bool EXACT>
__device__ __forceinline__ void tile_gather(const PfArgs<R> &a, const TilePlane<R> &lo, const TilePlane<R> &mid,
                                            const TilePlane<R> &hi, int tx, int ty, int gx, int gy, int gz, int n,
                                            R *lap, int lst)
{
    using T = TileShape<TX, TY>;
    const int h0 = (ty + 1) * T::HX + tx + 1;
    const int co[3] = {gx, gy, gz};
    const int dh[3] = {1, T::HX, 0};
    for (int g = 0; g < n; g++) lap[g * lst] = (R)0;
    /* faces from below without wrap, descending direction */
#pragma unroll
    for (int e = DIM - 1; e >= 0; e--) {
        if (co[e] > 0) {
            if (e == 2) tile_face<T::HC, R, EXACT>(a, mid, h0, n, lo, h0, lap, lst, false);
            else tile_face<T::HC, R, EXACT>(a, mid, h0, n, mid, h0 - dh[e], lap, lst, false);
        }
    }
    /* own faces, ascending direction */
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        if (co[d] < a.res[d] - 1 || (a.per[d] && a.res[d] > 1)) {
            if (d == 2) tile_face<T::HC, R, EXACT>(a, mid, h0, n, hi, h0, lap, lst, true);
            else tile_face<T::HC, R, EXACT>(a, mid, h0, n, mid, h0 + dh[d], lap, lst, true);
        }
    }
    /* faces wrapping around from above, ascending direction */
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        if (co[d] == 0 && a.per[d] && a.res[d] > 1) {
            if (d == 2) tile_face<T::HC, R, EXACT>(a, mid, h0, n, lo, h0, lap, lst, false);
            else tile_face<T::HC, R, EXACT>(a, mid, h0, n, mid, h0 - dh[d], lap, lst, false);
        }
    }
}

}  // namespace cipher
