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
 *   1. lane = cell: active count and the cell's face-map words (as 32-bit
 *      halves, slots 0-7 and 8-15) into shared memory, one 16-bit tag (cell lane, slot) per item in slot-major
 *      order;
 *   2. lane = item: the slot's phase fraction and its Laplacian over the
 *      cell's 2*dim faces (absent or gated faces map every slot to 15);
 *      neighbour cells follow from the row's position (y and z offsets are
 *      the same for the whole row);
 *   3. lane = cell: the O(n) closed forms of the cell terms and all P
 *      slots of F (coalesced plane by plane).
 * Laplacians pass from phase 2 to phase 3 in a slot-major table with row
 * pitch 33, so that phase 3's lanes read distinct banks; phase 3 re-reads
 * the cell's phase fractions (coalesced, cached since phase 2).
 * The mixed path sums a Laplacian in direction order, not in the
 * reference's face order: the difference is FP32 rounding.
 * IX is the index type of plane offsets: int when every offset of the
 * domain fits (max(P, 2*dim) * stride < 2^31, all benchmark and batch
 * sizes), int64_t otherwise.
 */
__host__ __device__ constexpr size_t items_warp_bytes(int dim, int P)
{
    return ((size_t)32 * 2 * dim * 8 + (size_t)33 * P * 4 + (size_t)32 * P * 2 + 15) / 16 * 16;
}

__host__ __device__ constexpr size_t items_tile_bytes(int dim, int T, int P, int ix_bytes)
{
    return (void)ix_bytes, (size_t)(T / 32) * items_warp_bytes(dim, P);
}

/* whether a domain's plane offsets fit the 32-bit kernels */
__host__ __device__ inline bool items_fit_i32(int64_t stride, int P, int dim)
{
    const int64_t planes = P > 2 * dim ? P : 2 * dim;
    return planes * stride < ((int64_t)1 << 31) - 1;
}

template <int DIM, typename IX>
__device__ __forceinline__ void mixed_items_tile(const PfArgs<float> &a, const CellIndex &cix, unsigned char *smem)
{
    constexpr int ND = 2 * DIM;
    const int lane = threadIdx.x & 31, P = a.P;
    const IX S = (IX)a.stride;
    const float *phi = a.phi;
    unsigned char *ws = smem + (size_t)(threadIdx.x >> 5) * items_warp_bytes(DIM, P);
    uint32_t *sw = (uint32_t *)ws;                                /* [ND][2][32] face-map word halves */
    float *slap = (float *)(sw + ND * 64);                        /* [P][33] Laplacian, later the capillary force */
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
    if (n > 0) {
        const int co[3] = {cix.x, cix.y, cix.z};
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const bool wrap = a.per[d] && a.res[d] > 1;
            const bool lo = co[d] > 0 || wrap, hi = co[d] < a.res[d] - 1 || wrap;
            const uint64_t wl = lo ? __ldg(&a.maps[(IX)(2 * d) * S + c]) : ~0ull;
            const uint64_t wh = hi ? __ldg(&a.maps[(IX)(2 * d + 1) * S + c]) : ~0ull;
            sw[(4 * d + 0) * 32 + lane] = (uint32_t)wl;
            sw[(4 * d + 1) * 32 + lane] = (uint32_t)(wl >> 32);
            sw[(4 * d + 2) * 32 + lane] = (uint32_t)wh;
            sw[(4 * d + 3) * 32 + lane] = (uint32_t)(wh >> 32);
        }
    }
    /* items in slot-major order (slot 0 of every cell, then slot 1 of the
     * cells that have one, ...): consecutive lanes then gather neighbouring
     * cells of the same planes, which share sectors */
    const int maxn = __reduce_max_sync(0xffffffffu, n);
    const unsigned below = (1u << lane) - 1u;
    int total = 0;
    for (int k = 0; k < maxn; k++) {
        const unsigned m = __ballot_sync(0xffffffffu, n > k);
        if (n > k) itag[total + __popc(m & below)] = (uint16_t)(lane | k << 5);
        total += __popc(m);
    }
    __syncwarp();

    /* 2. items, kIPP per pass so that their loads are in flight together */
    const float coef = a.coef_f;
    const IX xlo_wrap = (IX)(a.res[0] - 1), xhi_wrap = -(IX)(a.res[0] - 1);
    for (int it = lane; it < total; it += 32 * kIPP) {
        int cl[kIPP], sl[kIPP];
        bool ok[kIPP];
        float l[kIPP];
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
            const float p = __ldg(&phi[(IX)sl[u] * S + cc]);
            const unsigned sh = 4u * (unsigned)(sl[u] & 7);
            const uint32_t *swh = sw + (sl[u] >> 3) * 32 + cl[u];   /* the word half holding slot sl */
            float pn[ND];
#pragma unroll
            for (int q = 0; q < ND; q++) {
                const int j = (int)((swh[q * 64] >> sh) & 15u);
                IX dq;
                if (q == 0) dq = x > 0 ? (IX)-1 : xlo_wrap;
                else if (q == 1) dq = x < a.res[0] - 1 ? (IX)1 : xhi_wrap;
                else dq = (q & 1) ? dhi[q >> 1] : dlo[q >> 1];
                pn[q] = j < P ? __ldg(&phi[(IX)j * S + cc + dq]) : p;
            }
            float acc = 0.0f;
#pragma unroll
            for (int q = 0; q < ND; q++) acc += pn[q] - p;
            l[u] = coef * acc;
        }
#pragma unroll
        for (int u = 0; u < kIPP; u++)
            if (ok[u]) slap[sl[u] * 33 + cl[u]] = l[u];
    }
    __syncwarp();

    /* 3. cell terms in FP32.  The sum of the capillary forces over the
     * cell's slots has a closed form in the slot sums:
     *   C = 8 (-sigma (n-1) A - tj/2 (n-2)(S1^2 - S2)) + L,   L = sum of Laplacians,
     * so one pass gives the sums and a second the forces and the active set */
    if (!cix.live) return;
    uint32_t act = 0;
    float nf = 0.0f, Caf = 0.0f;
    float *cl3 = slap + lane;        /* slot k at cl3[33 * k] */
    const float *cp3 = phi + c;      /* slot k at cp3[k * S] (cached since phase 2) */
    if (n > 1) {
        const float inv_w = a.inv_w_f, w_pi2 = a.w_pi2_f, sig = a.sig_f, tjh = a.tjh_f, mob = a.mob_f;
        float A = 0.0f, S1 = 0.0f, S2 = 0.0f, L = 0.0f;
        {
            const float *pp = cp3;
#pragma unroll 2
            for (int k = 0; k < n; k++, pp += S) {
                const float pk = __ldg(pp), lk = cl3[33 * k];
                A += pk * inv_w + lk * w_pi2;
                S1 += pk;
                S2 += pk * pk;
                L += lk;
            }
        }
        const float fn = (float)n;
        const float C = 8.0f * (-sig * (fn - 1.0f) * A - tjh * (fn - 2.0f) * (S1 * S1 - S2)) + L;
        const float *pp = cp3;
#pragma unroll 2
        for (int k = 0; k < n; k++, pp += S) {
            const float pk = __ldg(pp), lk = cl3[33 * k];
            const float ak = pk * inv_w + lk * w_pi2;
            const float o1 = S1 - pk, o2 = S2 - pk * pk;
            const float cap = 8.0f * (-sig * (A - ak) - tjh * (o1 * o1 - o2)) + lk;
            cl3[33 * k] = cap;
            const float u = mob * (fn * cap - C);
            const bool on = (pk > a.tol_gt && pk < a.tol1_lt) || (pk < a.tol_lt && u > 0.0f) ||
                            (pk > a.tol1_gt && u < 0.0f);
            act |= (uint32_t)on << k;
            nf += on ? 1.0f : 0.0f;
            Caf += on ? cap : 0.0f;
        }
    }
    /* F = m (nact cap - Ca) / nact on the active slots, 0 elsewhere; slots
     * at or above the row's largest count are 0 for every lane */
    const float scale = act ? a.mob_f * __frcp_rn(nf) : 0.0f;
    float *fp = a.fphi + c;
    int m = 0;
#pragma unroll 2
    for (; m < maxn; m++) {
        float vv = 0.0f;
        if (act >> m & 1u) vv = scale * fmaf(nf, cl3[33 * m], -Caf);
        *fp = vv;
        fp += S;
    }
#pragma unroll 2
    for (; m < P; m++) {
        *fp = 0.0f;
        fp += S;
    }
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = (float)tr;
}

template <int DIM, typename IX>
__global__ void __launch_bounds__(kMixedBlock) k_rhs_pf_mixed_items(const PfArgs<float> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const CellIndex ci = cell_index<kBX, kBY>(a.res, a.zbase);
    mixed_items_tile<DIM, IX>(a, ci, smem);
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
        if (SINGLE) mixed_items_tile<DIM, IX>(b.args[inst], ci, smem);
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

template <int DIM, int PM>
static void launch_pm(const PfArgs<float> &a, cudaStream_t s)
{
    dim3 grid((unsigned)((a.res[0] + kBX - 1) / kBX), (unsigned)((a.res[1] + kBY - 1) / kBY),
              (unsigned)(a.zcount > 0 ? a.zcount : a.res[2]));
    if (a.single) {
        if (items_fit_i32(a.stride, a.P, DIM)) {
            const size_t sm = items_tile_bytes(DIM, kMixedBlock, a.P, 4);
            if (allow_smem(k_rhs_pf_mixed_items<DIM, int>, sm) != cudaSuccess) return;
            k_rhs_pf_mixed_items<DIM, int><<<grid, kMixedBlock, sm, s>>>(a);
        } else {
            const size_t sm = items_tile_bytes(DIM, kMixedBlock, a.P, 8);
            if (allow_smem(k_rhs_pf_mixed_items<DIM, int64_t>, sm) != cudaSuccess) return;
            k_rhs_pf_mixed_items<DIM, int64_t><<<grid, kMixedBlock, sm, s>>>(a);
        }
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
    const size_t sm = SINGLE ? items_tile_bytes(DIM, kBX * by, b.pmax, (int)sizeof(IX))
                             : slot_columns_bytes(b.pmax, kBX * by, 4, true);
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

cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_dim<1>(a, s);
    else if (dim == 2) launch_dim<2>(a, s);
    else launch_dim<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
