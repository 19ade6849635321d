/*
 * poststep.cu - per-step active-set update on uniform grids, the part of
 * PostStep at src/cipher.c:869-974.
 *
 *   k_post_prune : project phi of every cell with n > 1 onto the Gibbs
 *                  simplex (src/utility.c:578-603), write it back, and store
 *                  the pruned set {id : phi > TOL} in a scratch plane set;
 *                  cells with n == 1 get phi = 1.
 *   k_post_union : superset = own pruned set U pruned sets of the face
 *                  neighbours (sorted merge, src/utility.c:195-230); keep phi
 *                  and EX of surviving phases, zero phi and initialise EX of
 *                  new phases (SitepotentialExplicit of the material's c0 at
 *                  the cell temperature), write the superset.  A superset above P raises
 *                  the cap flag and leaves that cell's set unchanged.
 *
 * The projection and the TOL test run in FP64 for both precisions, so the
 * phase sets are decided by the same arithmetic as the reference.
 */
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"
#include "models.cuh"

namespace cipher {

template <int PM, typename R>
__device__ __forceinline__ void post_prune_cell(const PostArgs<R> &a, int64_t c)
{
    const int64_t S = a.stride;
    int n = a.as[c];
    if (n < 1 || n > a.P) {
        atomicOr(a.err, ERR_BADSET);
        a.pruned[c] = 0;
        return;
    }
    if (n == 1) {
        a.phi[c] = (R)1.0;
        a.pruned[c] = 1;
        a.pruned[S + c] = a.as[S + c];
        return;
    }
    double phi[PM], s[PM];
    uint16_t ids[PM];
    /* every load of the cell issued together */
#pragma unroll
    for (int g = 0; g < PM; g++)
        if (g < n) {
            phi[g] = (double)a.phi[(int64_t)g * S + c];
            ids[g] = a.as[(int64_t)(1 + g) * S + c];
            s[g] = phi[g];
        }
    /* sort a copy in descending order (insertion sort; n <= 16) */
    for (int i = 1; i < n; i++) {
        double v = s[i];
        int j = i - 1;
        while (j >= 0 && s[j] < v) { s[j + 1] = s[j]; j--; }
        s[j + 1] = v;
    }
    double sum = 0.0, tmax = 0.0;
    bool found = false;
    for (int i = 0; i < n - 1; i++) {
        sum += s[i];
        tmax = (sum - 1.0) / ((double)(i + 1));
        if (tmax >= s[i + 1]) { found = true; break; }
    }
    if (!found) tmax = (sum + s[n - 1] - 1.0) / ((double)n);
    int np = 0;
#pragma unroll
    for (int g = 0; g < PM; g++) {
        if (g < n) {
            double v = phi[g] - tmax > 0.0 ? phi[g] - tmax : 0.0;
            a.phi[(int64_t)g * S + c] = (R)v;
            if (v > CIPHER_TOL) {
                a.pruned[(int64_t)(1 + np) * S + c] = ids[g];
                np++;
            }
        }
    }
    a.pruned[c] = (uint16_t)np;
}

template <int PM, typename R>
__global__ void __launch_bounds__(256, 4) k_post_prune(const PostArgs<R> a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    post_prune_cell<PM, R>(a, c);
}

/* out = a U b (sorted); returns the size, or P+1 if it would exceed P */
template <int PM>
__device__ __forceinline__ int merge_union(const uint16_t *sa, int na, const uint16_t *pl, int64_t S, int64_t nb,
                                           int nbn, uint16_t *out, int P)
{
    int i = 0, j = 0, n = 0;
    uint16_t b = nbn > 0 ? pl[S + nb] : 0;
    while (i < na || j < nbn) {
        uint16_t v;
        if (j >= nbn || (i < na && sa[i] < b)) {
            v = sa[i++];
        } else if (i >= na || b < sa[i]) {
            v = b;
            j++;
            if (j < nbn) b = pl[(int64_t)(1 + j) * S + nb];
        } else {
            v = sa[i++];
            j++;
            if (j < nbn) b = pl[(int64_t)(1 + j) * S + nb];
        }
        if (n >= P) return P + 1;
        out[n++] = v;
    }
    return n;
}

/* write cell c's superset sup[0..ns): phi and EX of surviving phases move
 * to their new slots, new phases start at phi = 0 and EX =
 * SitepotentialExplicit(c0, T of the cell) (src/cipher.c:947-973) */
template <int PM, typename R>
__device__ __forceinline__ void post_write_cell(const PostArgs<R> &a, int64_t c, int n, int ns, const uint16_t *sup)
{
    const int64_t S = a.stride;
    /* old (unpruned) set of this cell: phi survives for phases in the superset */
    uint16_t old[PM];
    for (int k = 0; k < n; k++) old[k] = a.as[(int64_t)(1 + k) * S + c];
    R phiss[PM];
    int from[PM];
    for (int g = 0; g < ns; g++) { phiss[g] = (R)0; from[g] = -1; }
    {
        int i = 0, j = 0;
        while (i < n && j < ns) {
            if (old[i] == sup[j]) { from[j] = i; i++; j++; }
            else if (old[i] < sup[j]) i++;
            else j++;
        }
    }
    for (int g = 0; g < ns; g++)
        if (from[g] >= 0) phiss[g] = a.phi[(int64_t)from[g] * S + c];
    if (a.S > 0) {
        double exss[PM * 2 * CIPHER_MAXCP];
        const double T = (double)a.tm[c];
        for (int g = 0; g < ns; g++) {
            if (from[g] >= 0) {
                for (int q = 0; q < a.S; q++) exss[g * a.S + q] = a.ex[(int64_t)(from[g] * a.S + q) * S + c];
            } else if (a.chem.mat) {
                /* slots past the phase's own sites are never read; they start at 0 */
                const cipher_material &mat = material_of(a.chem, sup[g]);
                for (int q = 0; q < a.S; q++) exss[g * a.S + q] = 0.0;
                sitepot_explicit(a.chem, sup[g], mat.c0, T, &exss[g * a.S]);
            } else {
                for (int q = 0; q < a.S; q++) exss[g * a.S + q] = 0.0;
            }
        }
        for (int g = 0; g < ns; g++)
            for (int q = 0; q < a.S; q++) a.ex[(int64_t)(g * a.S + q) * S + c] = exss[g * a.S + q];
    }
    for (int g = 0; g < ns; g++) a.phi[(int64_t)g * S + c] = phiss[g];
    a.as[c] = (uint16_t)ns;
    for (int g = 0; g < ns; g++) a.as[(int64_t)(1 + g) * S + c] = sup[g];
}

/* union of an adapted mesh's cell with its listed neighbours' pruned sets
 * (src/cipher.c:930-945; the union does not depend on their order) */
template <int PM, typename R>
__device__ __forceinline__ void post_union_listed(const PostArgs<R> &a, int64_t c)
{
    const int64_t S = a.stride;
    const int n = a.as[c];
    int ns = a.pruned[c];
    if (n < 1 || n > a.P || ns < 1 || ns > a.P) return;   /* flagged by k_post_prune */
    uint16_t sup[PM], tmp[PM];
    for (int k = 0; k < ns; k++) sup[k] = a.pruned[(int64_t)(1 + k) * S + c];
    for (int32_t e = a.fl.start[c]; e < a.fl.start[c + 1]; e++) {
        const int64_t nb = a.fl.nbr[e] & 0x7fffffff;
        if (nb == c) continue;
        int nbn = a.pruned[nb];
        if (nbn > a.P) nbn = a.P;
        const int m = merge_union<PM>(sup, ns, a.pruned, S, nb, nbn, tmp, a.P);
        if (m > a.P) {
            atomicOr(a.err, ERR_CAP);
            return;
        }
        for (int k = 0; k < m; k++) sup[k] = tmp[k];
        ns = m;
    }
    post_write_cell<PM, R>(a, c, n, ns, sup);
}

template <int PM, typename R>
__global__ void __launch_bounds__(256) k_post_union_listed(const PostArgs<R> a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    post_union_listed<PM, R>(a, c);
}

/* ------------------------------------------------------------------ */
/* uniform grids: one warp per row of 32 cells, sets staged in shared   */
/* memory                                                               */
/* ------------------------------------------------------------------ */
/*
 * The union and the face maps of a cell need the sets of its 2*dim face
 * neighbours.  A warp owns a row of 32 consecutive x cells of grid line
 * (y, z) and stages, plane by plane with coalesced loads, the sets (count,
 * then ids) of its own row and of the rows at y-1, y+1, z-1, z+1 in shared
 * memory, plus the two cells just outside the row along x.  Every merge then
 * reads shared memory instead of chaining dependent global loads.  Blocks are
 * 4 warps on 4 consecutive y rows.
 */
constexpr int kPostRowWarps = 4;

/* staged rows: 0 own, 1 y-1, 2 y+1, 3 z-1, 4 z+1; entries [row][k][32], k = 0
 * count, 1..P ids; then two halo cells [2][P+1] */
__host__ __device__ constexpr size_t post_stage_elems(int P) { return (size_t)5 * (P + 1) * 32 + 2 * (P + 1); }

/* a warp's slice of shared memory, each region on a 16-byte boundary:
 * staged sets (uint16), then the per-lane work columns - two uint16
 * superset columns [P][32] (union) or one uint32 map-word column [P][32]
 * (maps) - then an 8-byte column [P][32] (the union's old phase fractions) */
__host__ __device__ constexpr size_t post_stage_bytes(int P) { return (post_stage_elems(P) * 2 + 15) / 16 * 16; }
__host__ __device__ constexpr size_t post_work_offset(int P) { return post_stage_bytes(P); }
__host__ __device__ constexpr size_t post_old_offset(int P) { return post_stage_bytes(P) + (size_t)P * 32 * 4; }
__host__ __device__ constexpr size_t post_row_warp_bytes(int P) { return post_old_offset(P) + (size_t)P * 32 * 8; }
/* the face-map kernel needs no old-phase column */
__host__ __device__ constexpr size_t maps_row_warp_bytes(int P) { return post_old_offset(P); }

/* 16-byte asynchronous copies global -> shared (no registers held) */
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

struct RowCells {
    int x0, y, z;          /* row origin */
    int x;                 /* this lane's x */
    bool live;
    int64_t c;             /* this lane's cell */
    int nlive;             /* live lanes of the row */
};

template <int DIM>
__device__ __forceinline__ bool row_of(const int *res, int64_t rb, int wib, RowCells &r)
{
    const int nxs = (res[0] + 31) >> 5;
    const int nyb = (res[1] + kPostRowWarps - 1) / kPostRowWarps;
    const int xs = (int)(rb % nxs);
    const int64_t rest = rb / nxs;
    r.y = (int)(rest % nyb) * kPostRowWarps + wib;
    r.z = (int)(rest / nyb);
    if (r.y >= res[1] || r.z >= res[2]) return false;
    r.x0 = xs * 32;
    r.x = r.x0 + (int)(threadIdx.x & 31);
    r.live = r.x < res[0];
    r.nlive = res[0] - r.x0 < 32 ? res[0] - r.x0 : 32;
    r.c = (int64_t)r.x + (int64_t)res[0] * ((int64_t)r.y + (int64_t)res[1] * r.z);
    return true;
}

/* cell offset of the neighbour row along d (1: y, 2: z) on `side`, or
 * INT64_MIN when that row is absent (non-periodic boundary, or a
 * dimension of one cell) */
__device__ __forceinline__ int64_t row_offset(const int *res, const int *per, const RowCells &r, int d, int side)
{
    const int co = d == 1 ? r.y : r.z;
    const int64_t st = d == 1 ? (int64_t)res[0] : (int64_t)res[0] * res[1];
    if (side == 0) {
        if (co > 0) return -st;
        if (per[d] && res[d] > 1) return (int64_t)(res[d] - 1) * st;
    } else {
        if (co < res[d] - 1) return st;
        if (per[d] && res[d] > 1) return -(int64_t)(res[d] - 1) * st;
    }
    return INT64_MIN;
}

/* x of the lower / upper x neighbour of x, or -1 */
__device__ __forceinline__ int x_nb(const int *res, const int *per, int x, int side)
{
    if (side == 0) return x > 0 ? x - 1 : (per[0] && res[0] > 1 ? res[0] - 1 : -1);
    return x < res[0] - 1 ? x + 1 : (per[0] && res[0] > 1 ? 0 : -1);
}

/* stage the sets held in planes (count plane, then P id planes, stride S) of
 * the row, its neighbour rows and its two outer x neighbours.  When rows are
 * whole 32-cell segments (res[0] a multiple of 32, so every row segment of a
 * plane is 64 bytes on a 16-byte boundary: planes start on 256-byte
 * boundaries and strides are multiples of 128) every plane of every row is
 * copied with 16-byte asynchronous copies, all in flight together;
 * otherwise a row's loads are issued together (unrolled to PM) before they
 * are stored.  Staged counts are the raw counts; readers clamp them to P. */
template <int DIM, int PM>
__device__ __forceinline__ void stage_row_sets(const uint16_t *planes, int64_t S, int P, const int *res, const int *per,
                                               const RowCells &r, uint16_t *st, bool *row_present)
{
    const int lane = threadIdx.x & 31;
    const int P1 = P + 1;
    /* whole 64-byte row segments on 16-byte boundaries (checked, not assumed) */
    const bool bulk = (res[0] & 31) == 0 && ((uintptr_t)planes & 15) == 0 && (S & 7) == 0;
    if (bulk) {
        const int64_t crow = r.c - lane;          /* first cell of the row */
        for (int row = 0; row < 5; row++) {
            int64_t off = 0;
            bool present = row == 0;
            if (row > 0) {
                const int d = (row + 1) >> 1;
                if (d < DIM) {
                    off = row_offset(res, per, r, d, (row + 1) & 1);
                    present = off != INT64_MIN;
                }
            }
            row_present[row] = present;
            if (!present) continue;
            uint16_t *rs = st + (size_t)row * P1 * 32;
            const uint16_t *src = planes + crow + off;
            for (int j = lane; j < P1 * 4; j += 32) {
                const int k = j >> 2, ch = j & 3;
                cp_async16(rs + k * 32 + ch * 8, src + (int64_t)k * S + ch * 8);
            }
        }
    } else {
    for (int row = 0; row < 5; row++) {
        int64_t off = 0;
        bool present = row == 0;
        if (row > 0) {
            const int d = (row + 1) >> 1;           /* 1,2 -> y ; 3,4 -> z */
            if (d < DIM) {
                off = row_offset(res, per, r, d, (row + 1) & 1);
                present = off != INT64_MIN;
            }
        }
        row_present[row] = present;
        if (!present) continue;
        uint16_t *rs = st + (size_t)row * P1 * 32;
        const int64_t cc = r.c + off;
        int n = r.live ? (int)planes[cc] : 0;
        if (n > P) n = P;
        rs[lane] = (uint16_t)n;
        uint16_t v[PM];
#pragma unroll
        for (int k = 0; k < PM; k++)
            if (k < n) v[k] = planes[(int64_t)(1 + k) * S + cc];
#pragma unroll
        for (int k = 0; k < PM; k++)
            if (k < n) rs[(1 + k) * 32 + lane] = v[k];
    }
    }
    /* the lower x neighbour of the first lane and the upper one of the last
     * live lane, when they lie outside the row */
    uint16_t *halo = st + (size_t)5 * P1 * 32;
    if (lane < 2) {
        const int xl = lane == 0 ? r.x0 : r.x0 + r.nlive - 1;
        const int xn = x_nb(res, per, xl, lane);
        uint16_t *h = halo + lane * P1;
        h[0] = 0;
        if (xn >= 0 && (xn < r.x0 || xn >= r.x0 + r.nlive)) {
            const int64_t cc = r.c - (r.x - xn);
            int n = planes[cc];
            if (n > P) n = P;
            h[0] = (uint16_t)n;
            uint16_t v[PM];
#pragma unroll
            for (int k = 0; k < PM; k++)
                if (k < n) v[k] = planes[(int64_t)(1 + k) * S + cc];
#pragma unroll
            for (int k = 0; k < PM; k++)
                if (k < n) h[1 + k] = v[k];
        }
    }
    if (bulk) cp_async_wait_all();
    __syncwarp();
}

/* the staged set of face neighbour q (2d + side) of this lane: its count
 * (0 when absent), the address of its first id and the id stride; `self`
 * tells that the neighbour is the cell itself (a periodic dimension of one
 * cell along x) */
template <int DIM>
__device__ __forceinline__ int staged_nb(const uint16_t *st, int P, const int *res, const int *per, const RowCells &r,
                                         const bool *row_present, int q, const uint16_t *&ids, int &stride)
{
    const int lane = threadIdx.x & 31;
    const int P1 = P + 1;
    const int d = q >> 1, side = q & 1;
    if (d == 0) {
        const int xn = x_nb(res, per, r.x, side);
        if (xn < 0 || xn == r.x) return 0;
        if (xn >= r.x0 && xn < r.x0 + r.nlive) {
            const uint16_t *rs = st + (xn - r.x0);
            ids = rs + 32;
            stride = 32;
            return rs[0] < P ? rs[0] : P;
        }
        const uint16_t *h = st + (size_t)5 * P1 * 32 + side * P1;   /* only the first / last lane gets here */
        ids = h + 1;
        stride = 1;
        return h[0];
    }
    const int row = 2 * d - 1 + side;
    if (!row_present[row]) return 0;
    const uint16_t *rs = st + (size_t)row * P1 * 32 + lane;
    ids = rs + 32;
    stride = 32;
    return rs[0] < P ? rs[0] : P;
}

/* union of this lane's pruned set with its face neighbours' (all staged).
 * EX: the state has explicit site potentials to move or initialise (the
 * per-cell form with its local tables); without them only phase fractions
 * move, through this lane's shared columns. */
template <int DIM, int PM, typename R, bool EX>
__device__ __forceinline__ void post_union_row(const PostArgs<R> &a, int64_t rb, unsigned char *wsm)
{
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    RowCells r;
    if (!row_of<DIM>(a.res, rb, wib, r)) return;           /* whole warp */
    const int P = a.P;
    uint16_t *st = (uint16_t *)wsm;
    uint16_t *supA = (uint16_t *)(wsm + post_work_offset(P)), *supB = supA + P * 32;
    bool present[5];
    stage_row_sets<DIM, PM>(a.pruned, a.stride, P, a.res, a.per, r, st, present);
    if (!r.live) return;
    const int n = a.as[r.c];
    int ns = st[lane];
    if (n < 1 || n > P || ns < 1 || ns > P) return;       /* flagged by k_post_prune */
    for (int k = 0; k < ns; k++) supA[k * 32 + lane] = st[(1 + k) * 32 + lane];
    uint16_t *cur = supA + lane, *nxt = supB + lane;
    for (int q = 0; q < 2 * DIM; q++) {
        const uint16_t *ids;
        int stride;
        const int nbn = staged_nb<DIM>(st, P, a.res, a.per, r, present, q, ids, stride);
        if (nbn == 0) continue;
        /* sorted merge cur U nb -> nxt */
        int i = 0, j = 0, m = 0;
        bool over = false;
        while (i < ns || j < nbn) {
            const uint16_t u = i < ns ? cur[i * 32] : 0xffff, v = j < nbn ? ids[j * stride] : 0xffff;
            uint16_t w;
            if (j >= nbn || (i < ns && u < v)) { w = u; i++; }
            else if (i >= ns || v < u) { w = v; j++; }
            else { w = u; i++; j++; }
            if (m >= P) { over = true; break; }
            nxt[m++ * 32] = w;
        }
        if (over) {
            atomicOr(a.err, ERR_CAP);
            return;
        }
        uint16_t *t = cur;
        cur = nxt;
        nxt = t;
        ns = m;
    }
    if (EX) {
        uint16_t sup[PM];
        for (int k = 0; k < ns; k++) sup[k] = cur[k * 32];
        post_write_cell<PM, R>(a, r.c, n, ns, sup);
        return;
    }
    /* phase fractions only: the cell's old ids and phi go to this lane's
     * own shared columns (loads four at a time); then the superset is
     * written slot by slot (survivors keep phi, new phases get 0) */
    const int64_t S = a.stride;
    uint16_t *oid = nxt;                                  /* the free superset column */
    double *oph = (double *)(wsm + post_old_offset(P)) + lane;
    for (int k0 = 0; k0 < n; k0 += 4) {
        R v[4];
        uint16_t id[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (k0 + j < n) { id[j] = a.as[(int64_t)(1 + k0 + j) * S + r.c]; v[j] = a.phi[(int64_t)(k0 + j) * S + r.c]; }
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (k0 + j < n) { oid[(k0 + j) * 32] = id[j]; oph[(k0 + j) * 32] = (double)v[j]; }
    }
    /* a superset equal to the old set changes nothing: every phase keeps its
     * slot and its (projected) phase fraction */
    if (ns == n) {
        bool same = true;
        for (int g = 0; g < ns && same; g++) same = cur[g * 32] == oid[g * 32];
        if (same) return;
    }
    int i = 0;
    for (int g = 0; g < ns; g++) {
        const uint16_t idg = cur[g * 32];
        while (i < n && oid[i * 32] < idg) i++;
        const R v = (i < n && oid[i * 32] == idg) ? (R)oph[i * 32] : (R)0;
        a.phi[(int64_t)g * S + r.c] = v;
    }
    a.as[r.c] = (uint16_t)ns;
    for (int g = 0; g < ns; g++) a.as[(int64_t)(1 + g) * S + r.c] = cur[g * 32];
}

template <int DIM, int PM, typename R, bool EX>
__global__ void __launch_bounds__(32 * kPostRowWarps) k_post_union_rows(const PostArgs<R> a, int64_t rb0)
{
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char *wsm = smem + (size_t)(threadIdx.x >> 5) * post_row_warp_bytes(a.P);
    post_union_row<DIM, PM, R, EX>(a, rb0 + blockIdx.x, wsm);
}

/*
 * Face maps (cipher_b200.h, MAP) of this lane's cell: one 32-bit word per
 * active slot, nibble q = 2d + side holding the slot of the same phase in
 * the neighbour across face q, or 15 where the neighbour lacks it or the
 * face's L cell (the lower one, as the reference enumerates faces (c, c+e_d))
 * fails the phase-flux gate of src/cipher.c:277.  Bad sets raise
 * ERR_BADSET.
 */
template <int DIM, int PM, typename R>
__device__ __forceinline__ void build_maps_row(const PostArgs<R> &a, int64_t rb, unsigned char *wsm)
{
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    RowCells r;
    if (!row_of<DIM>(a.res, rb, wib, r)) return;
    const int P = a.P;
    const int64_t S = a.stride;
    uint16_t *st = (uint16_t *)wsm;
    uint32_t *mw = (uint32_t *)(wsm + post_work_offset(P));
    bool present[5];
    stage_row_sets<DIM, PM>(a.as, S, P, a.res, a.per, r, st, present);
    if (!r.live) return;
    const int n = a.as[r.c];
    bool ok = n >= 1 && n <= P;
    const uint16_t *own = st + 32 + lane;
    if (ok && a.npf > 0)
        for (int k = 0; k < n; k++)
            if (own[k * 32] >= a.npf) ok = false;
    if (!ok) {
        atomicOr(a.err, ERR_BADSET);
        return;
    }
    uint32_t *w = mw + lane;
    for (int k = 0; k < n; k++) w[k * 32] = 0xffffffffu;
    const bool gate_self = n > 1 || own[0] > 1;
    for (int q = 0; q < 2 * DIM; q++) {
        const uint16_t *ids;
        int stride;
        const int nn = staged_nb<DIM>(st, P, a.res, a.per, r, present, q, ids, stride);
        if (nn < 1) continue;
        const bool gate = (q & 1) ? gate_self : (nn > 1 || ids[0] > 1);
        if (!gate) continue;
        const unsigned sh = 4u * (unsigned)q;
        int i = 0, j = 0;
        while (i < n && j < nn) {
            const uint16_t u = own[i * 32], v = ids[j * stride];
            if (u == v) {
                w[i * 32] = (w[i * 32] & ~(15u << sh)) | ((uint32_t)j << sh);
                i++;
                j++;
            } else if (u < v) {
                i++;
            } else {
                j++;
            }
        }
    }
    for (int k = 0; k < n; k++) a.maps[(int64_t)k * S + r.c] = w[k * 32];
}

template <int DIM, int PM, typename R>
__global__ void __launch_bounds__(32 * kPostRowWarps) k_build_maps_rows(const PostArgs<R> a, int64_t rb0)
{
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char *wsm = smem + (size_t)(threadIdx.x >> 5) * maps_row_warp_bytes(a.P);
    build_maps_row<DIM, PM, R>(a, rb0 + blockIdx.x, wsm);
}

/* the kernels' slot arrays are sized by a bucket of P: 4, 8, 12 or 16 */
template <typename F>
__host__ inline cudaError_t with_pm(int P, F f)
{
    if (P <= 4) return f(std::integral_constant<int, 4>());
    if (P <= 8) return f(std::integral_constant<int, 8>());
    if (P <= 12) return f(std::integral_constant<int, 12>());
    return f(std::integral_constant<int, 16>());
}
template <typename F>
__host__ inline cudaError_t with_dim(int dim, F f)
{
    if (dim == 1) return f(std::integral_constant<int, 1>());
    if (dim == 2) return f(std::integral_constant<int, 2>());
    return f(std::integral_constant<int, 3>());
}

/* row blocks of a grid (4 rows of 32 cells each) and of its z-planes [z0, z1) */
__host__ __device__ inline int64_t row_blocks_per_plane(const int *res)
{
    return (int64_t)((res[0] + 31) >> 5) * ((res[1] + kPostRowWarps - 1) / kPostRowWarps);
}
__host__ __device__ inline int64_t row_blocks(const int *res) { return row_blocks_per_plane(res) * res[2]; }
int64_t post_row_blocks(const int *res) { return row_blocks(res); }

template <typename R>
static cudaError_t launch_maps(const PostArgs<R> &a, int dim, int64_t z0, int64_t z1, cudaStream_t s)
{
    if (!a.maps || z1 <= z0) return cudaSuccess;
    const int64_t per = row_blocks_per_plane(a.res);
    const unsigned blocks = (unsigned)((z1 - z0) * per);
    const size_t sm = kPostRowWarps * maps_row_warp_bytes(a.P);
    return with_dim(dim, [&](auto D) {
        return with_pm(a.P, [&](auto PMC) {
            k_build_maps_rows<D(), PMC(), R><<<blocks, 32 * kPostRowWarps, sm, s>>>(a, z0 * per);
            return cudaGetLastError();
        });
    });
}

cudaError_t launch_build_maps(const PostArgs<double> &a, int dim, cudaStream_t s) { return launch_maps(a, dim, 0, a.res[2], s); }
cudaError_t launch_build_maps(const PostArgs<float> &a, int dim, cudaStream_t s) { return launch_maps(a, dim, 0, a.res[2], s); }
/* cells [c0, c1) must be whole z-planes of a 3D grid */
cudaError_t launch_build_maps_range(const PostArgs<double> &a, int dim, int64_t c0, int64_t c1, cudaStream_t s)
{
    const int64_t plane = (int64_t)a.res[0] * a.res[1];
    return launch_maps(a, dim, c0 / plane, (c1 + plane - 1) / plane, s);
}
cudaError_t launch_build_maps_range(const PostArgs<float> &a, int dim, int64_t c0, int64_t c1, cudaStream_t s)
{
    const int64_t plane = (int64_t)a.res[0] * a.res[1];
    return launch_maps(a, dim, c0 / plane, (c1 + plane - 1) / plane, s);
}

/* batched: block k of a list belongs to the domain whose range holds k */
__device__ __forceinline__ int batch_domain_of(const int64_t *start, int n, int64_t k)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&start[mid]) <= k) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int PM, typename R>
__global__ void __launch_bounds__(256) k_post_prune_batched(const BatchPost<R> b)
{
    const int inst = batch_domain_of(b.block_start, b.n, blockIdx.x);
    if (!b.active[inst]) return;
    const PostArgs<R> &a = b.args[inst];
    const int64_t c = (int64_t)(blockIdx.x - b.block_start[inst]) * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    post_prune_cell<PM, R>(a, c);
}

template <int DIM, int PM, typename R, bool EX>
__global__ void __launch_bounds__(32 * kPostRowWarps) k_post_union_rows_batched(const BatchPost<R> b)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int inst = batch_domain_of(b.row_start, b.n, blockIdx.x);
    if (!b.active[inst]) return;
    const PostArgs<R> &a = b.args[inst];
    if ((a.S > 0) != EX) return;                          /* the other kind's launch takes it */
    unsigned char *wsm = smem + (size_t)(threadIdx.x >> 5) * post_row_warp_bytes(b.pmax);
    post_union_row<DIM, PM, R, EX>(a, blockIdx.x - b.row_start[inst], wsm);
}

template <int DIM, int PM, typename R>
__global__ void __launch_bounds__(32 * kPostRowWarps) k_build_maps_rows_batched(const BatchPost<R> b)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int inst = batch_domain_of(b.row_start, b.n, blockIdx.x);
    if (!b.active[inst]) return;
    const PostArgs<R> &a = b.args[inst];
    if (!a.maps) return;
    unsigned char *wsm = smem + (size_t)(threadIdx.x >> 5) * post_row_warp_bytes(b.pmax);
    build_maps_row<DIM, PM, R>(a, blockIdx.x - b.row_start[inst], wsm);
}

template <typename R>
static cudaError_t launch_post_batched(const BatchPost<R> &b, int dim, cudaStream_t s)
{
    if (b.total < 1) return cudaSuccess;
    cudaError_t e = with_pm(b.pmax, [&](auto PMC) {
        k_post_prune_batched<PMC(), R><<<(unsigned)b.total, 256, 0, s>>>(b);
        return cudaGetLastError();
    });
    if (e != cudaSuccess) return e;
    const size_t sm = kPostRowWarps * post_row_warp_bytes(b.pmax);
    const unsigned rb = (unsigned)b.row_total;
    const unsigned bs = 32 * kPostRowWarps;
    return with_dim(dim, [&](auto D) {
        return with_pm(b.pmax, [&](auto PMC) {
            /* domains with and without site potentials: one launch each */
            k_post_union_rows_batched<D(), PMC(), R, false><<<rb, bs, sm, s>>>(b);
            k_post_union_rows_batched<D(), PMC(), R, true><<<rb, bs, sm, s>>>(b);
            k_build_maps_rows_batched<D(), PMC(), R><<<rb, bs, sm, s>>>(b);
            return cudaGetLastError();
        });
    });
}

cudaError_t launch_poststep_batched(const BatchPost<double> &b, int dim, cudaStream_t s) { return launch_post_batched(b, dim, s); }
cudaError_t launch_poststep_batched(const BatchPost<float> &b, int dim, cudaStream_t s) { return launch_post_batched(b, dim, s); }

template <typename R>
static cudaError_t launch_post(const PostArgs<R> &a, int dim, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((a.ncells + 255) / 256);
    cudaError_t e = with_pm(a.P, [&](auto PMC) {
        k_post_prune<PMC(), R><<<blocks, 256, 0, s>>>(a);
        return cudaGetLastError();
    });
    if (e != cudaSuccess) return e;
    if (a.fl.start) {
        /* adapted meshes: neighbours from the face lists, no face maps */
        k_post_union_listed<CIPHER_PMAX, R><<<blocks, 256, 0, s>>>(a);
        return cudaGetLastError();
    }
    const size_t sm = kPostRowWarps * post_row_warp_bytes(a.P);
    const unsigned rb = (unsigned)row_blocks(a.res);
    e = with_dim(dim, [&](auto D) {
        return with_pm(a.P, [&](auto PMC) {
            if (a.S > 0) k_post_union_rows<D(), PMC(), R, true><<<rb, 32 * kPostRowWarps, sm, s>>>(a, 0);
            else k_post_union_rows<D(), PMC(), R, false><<<rb, 32 * kPostRowWarps, sm, s>>>(a, 0);
            return cudaGetLastError();
        });
    });
    if (e != cudaSuccess) return e;
    return launch_maps(a, dim, 0, a.res[2], s);
}

cudaError_t launch_poststep(const PostArgs<double> &a, int dim, cudaStream_t s) { return launch_post(a, dim, s); }
cudaError_t launch_poststep(const PostArgs<float> &a, int dim, cudaStream_t s) { return launch_post(a, dim, s); }

}  // namespace cipher
