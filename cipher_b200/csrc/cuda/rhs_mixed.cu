/*
 * rhs_mixed.cu - FP32-mixed RHS of the multi-phase-field equation on uniform
 * grids for problems without chemistry (the FP64 version is
 * rhs_phasefield.cu; the equations are src/cipher.c:235-317 and 391-555).
 *
 * Phase fractions, the stencil and the interface terms are FP32 (storage and
 * arithmetic).  The single-interface kernel keeps every cell term in FP32;
 * the several-interface form accumulates the pair-rate reductions that
 * decide the active set and the constrained rate in FP64.  For a single
 * interface the pair and triple sums of the reference collapse to per-cell
 * sums:
 *   sum_{j != k} sigma*a_j              = sigma*(A - a_k)
 *   sum_{j<i; j,i != k} phi_j*phi_i    = ((S1-phi_k)^2 - (S2-phi_k^2))/2
 *   sum_{j != k} m*(cap_k - cap_j)     = m*(n*cap_k - C)
 * (A = sum a_j, S1 = sum phi_j, S2 = sum phi_j^2, C = sum cap_j), which
 * makes the cell terms O(n) instead of O(n^3).  Several interfaces use the
 * reference-order evaluation of pf_cell.cuh in FP32.  Accuracy against the
 * FP64 oracle on the same inputs: max|dF|/max|F| <= 1e-6 (tested).
 */
#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"
#include "pf_cell.cuh"

#ifndef CIPHER_MIXED_BX
#define CIPHER_MIXED_BX 32
#define CIPHER_MIXED_BY 4
#endif

namespace cipher {

constexpr int kBX = CIPHER_MIXED_BX, kBY = CIPHER_MIXED_BY, kMixedBlock = kBX * kBY;
#ifndef CIPHER_MIXED_IPP
#define CIPHER_MIXED_IPP 2
#endif
constexpr int kIPP = CIPHER_MIXED_IPP;   /* items per lane and pass in the items kernel */

/* ------------------------------------------------------------------ */
/* single interface: (cell, slot) items spread over a warp's lanes       */
/* ------------------------------------------------------------------ */
/*
 * Each warp owns one row of 32 consecutive cells (same y and z) and its own
 * slice of shared memory, so warps never wait for one another.  The face
 * gather, the bulk of the work, runs over the row's (cell, slot) items, so a
 * lane never idles while a neighbour lane walks a larger set:
 *   1. lane = cell: active count, and one 16-bit tag (cell lane, slot) per
 *      item in slot-major order;
 *   2. lane = item: the slot's phase fraction, its face-map word (one word
 *      per slot: the neighbour's slot across each face, 15 for absent or
 *      gated faces) and its Laplacian over the cell's 2*dim faces; neighbour
 *      cells follow from the row's position (y and z offsets are the same
 *      for the whole row);
 *   3. lane = cell: the O(n) closed forms of the cell terms and all P
 *      slots of F (coalesced plane by plane).
 * Laplacians pass from phase 2 to phase 3 in a slot-major table with row
 * pitch 33, so that phase 3's lanes read distinct banks; phase 3 re-reads
 * the cell's phase fractions (coalesced, cached since phase 2).
 * The mixed path sums a Laplacian in direction order, not in the
 * reference's face order: the difference is FP32 rounding.
 * IX is the index type of plane offsets: int when every offset of the
 * domain fits (max(P, 2*dim) * stride < 2^31, all benchmark and batch
 * sizes), int64_t otherwise.  R is the real type: float for the mixed
 * layout; double gives the same closed form on an FP64 state (the FP64
 * closed-form path, within rounding of the reference-order kernel).
 */
__host__ __device__ constexpr size_t items_warp_bytes(int P, int rbytes)
{
    return ((size_t)33 * P * rbytes + (size_t)32 * P * 2 + 15) / 16 * 16;
}

__host__ __device__ constexpr size_t items_tile_bytes(int T, int P, int rbytes)
{
    return (size_t)(T / 32) * items_warp_bytes(P, rbytes);
}

/* whether a domain's plane offsets fit the 32-bit kernels */
__host__ __device__ inline bool items_fit_i32(int64_t stride, int P, int dim)
{
    const int64_t planes = P > 2 * dim ? P : 2 * dim;
    return planes * stride < ((int64_t)1 << 31) - 1;
}

/* the closed-form constants in the kernel's real type: FP32 forms computed on
 * the host (with active-set thresholds equal to the double tests), or the
 * FP64 values themselves */
template <typename R>
struct ItemConsts {
    R coef, inv_w, w_pi2, sig, tjh, mob, tol_gt, tol1_lt, tol_lt, tol1_gt;
};

__device__ __forceinline__ ItemConsts<float> item_consts(const PfArgs<float> &a)
{
    return {a.coef_f, a.inv_w_f, a.w_pi2_f, a.sig_f, a.tjh_f, a.mob_f, a.tol_gt, a.tol1_lt, a.tol_lt, a.tol1_gt};
}

__device__ __forceinline__ ItemConsts<double> item_consts(const PfArgs<double> &a)
{
    const double pi2 = CIPHER_PI_D * CIPHER_PI_D;
    return {a.face_coef, 1.0 / a.wid0, a.wid0 / pi2, a.sig0, 0.5 * a.tj0, a.mob0,
            CIPHER_TOL, 1.0 - CIPHER_TOL, CIPHER_TOL, 1.0 - CIPHER_TOL};
}

__device__ __forceinline__ float item_rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double item_rcp(double x) { return 1.0 / x; }
__device__ __forceinline__ float item_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double item_fma(double a, double b, double c) { return fma(a, b, c); }

template <int DIM, typename IX, typename R>
__device__ __forceinline__ void items_tile(const PfArgs<R> &a, const CellIndex &cix, unsigned char *smem)
{
    constexpr int ND = 2 * DIM;
    const int lane = threadIdx.x & 31, P = a.P;
    const IX S = (IX)a.stride;
    const R *phi = a.phi;
    const ItemConsts<R> k = item_consts(a);
    unsigned char *ws = smem + (size_t)(threadIdx.x >> 5) * items_warp_bytes(P, (int)sizeof(R));
    R *slap = (R *)ws;                                            /* [P][33] Laplacian, later the capillary force */
    uint16_t *itag = (uint16_t *)(slap + 33 * P);                 /* [32*P] cell lane | slot << 5 */

    __syncwarp();                    /* the previous row's readers are done */
    /* 1. cells */
    const IX c = (IX)cix.c;
    const IX crow = c - (IX)lane;    /* cell of lane 0: the row is contiguous */
    const int xrow = cix.x - lane;
    int n = cix.live ? (int)__ldg(&a.as[c]) : 0;
    if (cix.live && (n < 1 || n > P)) {
        atomicOr(a.err, ERR_BADSET);
        n = 0;
    }
    /* neighbour offsets along y and z (the same for the row) */
    IX dlo[3] = {0, 0, 0}, dhi[3] = {0, 0, 0};
    {
        const int co[3] = {cix.x, cix.y, cix.z};
        IX st = 1;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const IX span = (IX)(a.res[d] - 1) * st;
            dlo[d] = co[d] > 0 ? -st : span;
            dhi[d] = co[d] < a.res[d] - 1 ? st : -span;
            st *= (IX)a.res[d];
        }
    }
    /* items in slot-major order (slot 0 of every cell, then slot 1 of the
     * cells that have one, ...): consecutive lanes then gather neighbouring
     * cells of the same planes, which share sectors */
    const int maxn = __reduce_max_sync(0xffffffffu, n);
    const unsigned below = (1u << lane) - 1u;
    int total = 0;
    for (int kk = 0; kk < maxn; kk++) {
        const unsigned m = __ballot_sync(0xffffffffu, n > kk);
        if (n > kk) itag[total + __popc(m & below)] = (uint16_t)(lane | kk << 5);
        total += __popc(m);
    }
    __syncwarp();

    /* 2. items, kIPP per pass so that their loads are in flight together; an
     * item's face-map word gives its neighbour slot across each face */
    const IX xlo_wrap = (IX)(a.res[0] - 1), xhi_wrap = -(IX)(a.res[0] - 1);
    for (int it = lane; it < total; it += 32 * kIPP) {
        int cl[kIPP], sl[kIPP];
        bool ok[kIPP];
        R l[kIPP];
#pragma unroll
        for (int u = 0; u < kIPP; u++) {
            ok[u] = it + 32 * u < total;
            const int tg = itag[ok[u] ? it + 32 * u : it];
            cl[u] = tg & 31;
            sl[u] = tg >> 5;
        }
#pragma unroll
        for (int u = 0; u < kIPP; u++) {
            const IX cc = crow + (IX)cl[u];
            const int x = xrow + cl[u];
            const R p = __ldg(&phi[(IX)sl[u] * S + cc]);
            const uint32_t w = __ldg(&a.maps[(IX)sl[u] * S + cc]);
            R pn[ND];
#pragma unroll
            for (int q = 0; q < ND; q++) {
                const int j = (int)((w >> (4 * q)) & 15u);
                IX dq;
                if (q == 0) dq = x > 0 ? (IX)-1 : xlo_wrap;
                else if (q == 1) dq = x < a.res[0] - 1 ? (IX)1 : xhi_wrap;
                else dq = (q & 1) ? dhi[q >> 1] : dlo[q >> 1];
                pn[q] = j < P ? __ldg(&phi[(IX)j * S + cc + dq]) : p;
            }
            R acc = (R)0;
#pragma unroll
            for (int q = 0; q < ND; q++) acc += pn[q] - p;
            l[u] = k.coef * acc;
        }
#pragma unroll
        for (int u = 0; u < kIPP; u++)
            if (ok[u]) slap[sl[u] * 33 + cl[u]] = l[u];
    }
    __syncwarp();

    /* 3. cell terms.  The sum of the capillary forces over the cell's slots
     * has a closed form in the slot sums:
     *   C = 8 (-sigma (n-1) A - tj/2 (n-2)(S1^2 - S2)) + L,   L = sum of Laplacians,
     * so one pass gives the sums and a second the forces and the active set */
    if (!cix.live) return;
    uint32_t act = 0;
    R nf = (R)0, Caf = (R)0;
    R *cl3 = slap + lane;            /* slot k at cl3[33 * k] */
    const R *cp3 = phi + c;          /* slot k at cp3[k * S] (cached since phase 2) */
    if (n > 1) {
        R A = (R)0, S1 = (R)0, S2 = (R)0, L = (R)0;
        {
            const R *pp = cp3;
#pragma unroll 2
            for (int kk = 0; kk < n; kk++, pp += S) {
                const R pk = __ldg(pp), lk = cl3[33 * kk];
                A += pk * k.inv_w + lk * k.w_pi2;
                S1 += pk;
                S2 += pk * pk;
                L += lk;
            }
        }
        const R fn = (R)n;
        const R C = (R)8 * (-k.sig * (fn - (R)1) * A - k.tjh * (fn - (R)2) * (S1 * S1 - S2)) + L;
        const R *pp = cp3;
#pragma unroll 2
        for (int kk = 0; kk < n; kk++, pp += S) {
            const R pk = __ldg(pp), lk = cl3[33 * kk];
            const R ak = pk * k.inv_w + lk * k.w_pi2;
            const R o1 = S1 - pk, o2 = S2 - pk * pk;
            const R cap = (R)8 * (-k.sig * (A - ak) - k.tjh * (o1 * o1 - o2)) + lk;
            cl3[33 * kk] = cap;
            const R u = k.mob * (fn * cap - C);
            const bool on = (pk > k.tol_gt && pk < k.tol1_lt) || (pk < k.tol_lt && u > (R)0) ||
                            (pk > k.tol1_gt && u < (R)0);
            act |= (uint32_t)on << kk;
            nf += on ? (R)1 : (R)0;
            Caf += on ? cap : (R)0;
        }
    }
    /* F = m (nact cap - Ca) / nact on the active slots, 0 elsewhere; slots
     * at or above the row's largest count are 0 for every lane */
    const R scale = act ? k.mob * item_rcp(nf) : (R)0;
    R *fp = a.fphi + c;
    int m = 0;
#pragma unroll 2
    for (; m < maxn; m++) {
        R vv = (R)0;
        if (act >> m & 1u) vv = scale * item_fma(nf, cl3[33 * m], -Caf);
        *fp = vv;
        fp += S;
    }
#pragma unroll 2
    for (; m < P; m++) {
        *fp = (R)0;
        fp += S;
    }
    R tr = (R)0;
    if (a.has_temp_rate) tr += (R)a.temp_rate;
    a.ftm[c] = tr;
}

template <int DIM, typename IX, typename R>
__global__ void __launch_bounds__(kMixedBlock) k_rhs_pf_items(const PfArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const CellIndex ci = cell_index<kBX, kBY>(a.res, a.zbase);
    items_tile<DIM, IX, R>(a, ci, smem);
}

/* one cell of the mixed RHS, several interfaces (reference-order cell terms in FP32) */
template <int DIM, int PM>
__device__ __forceinline__ void pf_mixed_multi_cell(const PfArgs<float> &a, const CellIndex &ci,
                                                    const SlotColumns<float> &sc)
{
    const int n = load_and_gather<DIM, PM, float, false, true>(a, ci, sc);
    const double T = n == 0 ? 0.0 : (double)a.tm[ci.c];
    cell_rates_ordered<float, false>(a, sc, n, ci.c, ci.live, T);
    if (!ci.live) return;
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[ci.c] = (float)tr;
}

template <int DIM, int PM>
__global__ void __launch_bounds__(kMixedBlock) k_rhs_pf_mixed_multi(const PfArgs<float> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const CellIndex ci = cell_index<kBX, kBY>(a.res, a.zbase);
    const SlotColumns<float> sc = slot_columns<float>(smem, a.P, blockDim.x, threadIdx.x, true);
    pf_mixed_multi_cell<DIM, PM>(a, ci, sc);
}

/* batched: a persistent grid walks the tiles of every domain of the batch */
template <int DIM, int PM, bool SINGLE, int BY, typename IX>
__global__ void __launch_bounds__(kBX * BY) k_rhs_pf_mixed_batched(const BatchTiles<float> b)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const SlotColumns<float> sc = slot_columns<float>(smem, b.pmax, blockDim.x, threadIdx.x, !SINGLE);
    for (int64_t t = blockIdx.x; t < b.total; t += gridDim.x) {
        int inst;
        const CellIndex ci = batch_cell_index<kBX, BY>(b, t, inst);
        if (!b.active[inst]) continue;          /* uniform across the block */
        if (SINGLE) items_tile<DIM, IX, float>(b.args[inst], ci, smem);
        else pf_mixed_multi_cell<DIM, PM>(b.args[inst], ci, sc);
    }
}

/* dynamic shared memory above the default 48 KB needs the kernel's opt-in;
 * it is set once per kernel and size (before any graph capture: the batch
 * driver's tile tuning launches every shape it later captures) */
template <typename K>
static cudaError_t allow_smem(K kernel, size_t bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    static std::mutex mu;
    static std::vector<std::pair<const void *, size_t>> done;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &d : done)
        if (d.first == (const void *)kernel && d.second >= bytes) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) done.push_back({(const void *)kernel, bytes});
    return e;
}

template <typename R, int DIM>
static cudaError_t launch_items(const PfArgs<R> &a, dim3 grid, cudaStream_t s)
{
    const size_t sm = items_tile_bytes(kMixedBlock, a.P, (int)sizeof(R));
    cudaError_t e;
    if (items_fit_i32(a.stride, a.P, DIM)) {
        if ((e = allow_smem(k_rhs_pf_items<DIM, int, R>, sm)) != cudaSuccess) return e;
        k_rhs_pf_items<DIM, int, R><<<grid, kMixedBlock, sm, s>>>(a);
    } else {
        if ((e = allow_smem(k_rhs_pf_items<DIM, int64_t, R>, sm)) != cudaSuccess) return e;
        k_rhs_pf_items<DIM, int64_t, R><<<grid, kMixedBlock, sm, s>>>(a);
    }
    return cudaGetLastError();
}

static dim3 items_grid(const int *res, int zcount)
{
    return dim3((unsigned)((res[0] + kBX - 1) / kBX), (unsigned)((res[1] + kBY - 1) / kBY),
                (unsigned)(zcount > 0 ? zcount : res[2]));
}

template <int DIM, int PM>
static void launch_pm(const PfArgs<float> &a, cudaStream_t s)
{
    const dim3 grid = items_grid(a.res, a.zcount);
    if (a.single) {
        launch_items<float, DIM>(a, grid, s);
    } else {
        size_t sm = slot_columns_bytes(a.P, kMixedBlock, 4, true);
        k_rhs_pf_mixed_multi<DIM, PM><<<grid, kMixedBlock, sm, s>>>(a);
    }
}

template <int DIM>
static void launch_dim(const PfArgs<float> &a, cudaStream_t s)
{
    if (a.P <= 4) launch_pm<DIM, 4>(a, s);
    else if (a.P <= 8) launch_pm<DIM, 8>(a, s);
    else if (a.P <= 12) launch_pm<DIM, 12>(a, s);
    else launch_pm<DIM, 16>(a, s);
}

template <int DIM, int PM, bool SINGLE, typename IX>
static cudaError_t launch_batched_ix(const BatchTiles<float> &b, int by, int grid, cudaStream_t s)
{
    const size_t sm = SINGLE ? items_tile_bytes(kBX * by, b.pmax, 4) : slot_columns_bytes(b.pmax, kBX * by, 4, true);
    cudaError_t e;
    if (by == 1) {
        if ((e = allow_smem(k_rhs_pf_mixed_batched<DIM, PM, SINGLE, 1, IX>, sm)) != cudaSuccess) return e;
        k_rhs_pf_mixed_batched<DIM, PM, SINGLE, 1, IX><<<grid, kBX, sm, s>>>(b);
    } else if (by == 2) {
        if ((e = allow_smem(k_rhs_pf_mixed_batched<DIM, PM, SINGLE, 2, IX>, sm)) != cudaSuccess) return e;
        k_rhs_pf_mixed_batched<DIM, PM, SINGLE, 2, IX><<<grid, kBX * 2, sm, s>>>(b);
    } else {
        if ((e = allow_smem(k_rhs_pf_mixed_batched<DIM, PM, SINGLE, 4, IX>, sm)) != cudaSuccess) return e;
        k_rhs_pf_mixed_batched<DIM, PM, SINGLE, 4, IX><<<grid, kBX * 4, sm, s>>>(b);
    }
    return cudaGetLastError();
}

/* the several-interface form keeps 64-bit indices; single-interface groups
 * take the 32-bit items kernel when every member fits */
template <int DIM, int PM, bool SINGLE>
static cudaError_t launch_batched_by(const BatchTiles<float> &b, int by, int grid, cudaStream_t s)
{
    if (SINGLE && b.i32) return launch_batched_ix<DIM, PM, SINGLE, int>(b, by, grid, s);
    return launch_batched_ix<DIM, PM, SINGLE, int64_t>(b, by, grid, s);
}

template <int DIM>
static cudaError_t launch_batched_dim(const BatchTiles<float> &b, int single, int by, int grid, cudaStream_t s)
{
    if (b.pmax <= 4) return single ? launch_batched_by<DIM, 4, true>(b, by, grid, s) : launch_batched_by<DIM, 4, false>(b, by, grid, s);
    if (b.pmax <= 8) return single ? launch_batched_by<DIM, 8, true>(b, by, grid, s) : launch_batched_by<DIM, 8, false>(b, by, grid, s);
    if (b.pmax <= 12) return single ? launch_batched_by<DIM, 12, true>(b, by, grid, s) : launch_batched_by<DIM, 12, false>(b, by, grid, s);
    return single ? launch_batched_by<DIM, 16, true>(b, by, grid, s) : launch_batched_by<DIM, 16, false>(b, by, grid, s);
}

cudaError_t launch_rhs_pf_batched(const BatchTiles<float> &b, int dim, int single, int by, int grid, cudaStream_t s)
{
    if (dim == 1) return launch_batched_dim<1>(b, single, by, grid, s);
    if (dim == 2) return launch_batched_dim<2>(b, single, by, grid, s);
    return launch_batched_dim<3>(b, single, by, grid, s);
}

/* the closed-form single-interface kernel on an FP64 state (FP64 arithmetic) */
cudaError_t launch_rhs_items_fp64(const PfArgs<double> &a, int dim, cudaStream_t s)
{
    const dim3 grid = items_grid(a.res, a.zcount);
    if (dim == 1) return launch_items<double, 1>(a, grid, s);
    if (dim == 2) return launch_items<double, 2>(a, grid, s);
    return launch_items<double, 3>(a, grid, s);
}

cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_dim<1>(a, s);
    else if (dim == 2) launch_dim<2>(a, s);
    else launch_dim<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
