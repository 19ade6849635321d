/*
 * rhs_phasefield.cu - FP64 RHS of the multi-phase-field equation on uniform
 * grids for problems without chemistry (every material `none` with a zero
 * reference energy, no segregation potential, D = 0): grain growth.
 *
 * Replaces, for that class of problems, RHSFunction (src/cipher.c:27-681):
 * the face loop (235-317) becomes a per-cell gather (pf_gather.cuh) and the
 * cell loop (391-664) runs in the same thread (pf_cell.cuh).
 *
 * Bit-identical to the reference: every value is formed by the same IEEE
 * operations in the same order (this unit is compiled with --fmad=false).
 * One thread per cell; all P slots of F are written (zero beyond n).
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
#include "order.cuh"

namespace cipher {

constexpr int kBX = 32, kBY = 2, kFp64Block = kBX * kBY;

/* one cell of the FP64 phase-field RHS (shared by the single-domain and the
 * batched kernels) */
template <int DIM, int PM, bool SINGLE>
__device__ __forceinline__ void pf_fp64_cell(const PfArgs<double> &a, const CellIndex &ci,
                                             const SlotColumns<double> &sc)
{
    const int n = load_and_gather<DIM, PM, double, true, !SINGLE>(a, ci, sc);
    const double T = (SINGLE || n == 0) ? 0.0 : a.tm[ci.c];
    cell_rates_ordered<double, SINGLE>(a, sc, n, ci.c, ci.live, T);
    if (!ci.live) return;
    /* temperature: no conductivity, latent or specific heat (src/cipher.c:558-568) */
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[ci.c] = tr;
}

template <int DIM, int PM, bool SINGLE>
__global__ void __launch_bounds__(kFp64Block) k_rhs_pf_fp64(const PfArgs<double> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const CellIndex ci = cell_index<kBX, kBY>(a.res, a.zbase);
    const SlotColumns<double> sc = slot_columns<double>(smem, a.P, blockDim.x, threadIdx.x, true);
    pf_fp64_cell<DIM, PM, SINGLE>(a, ci, sc);
}

/* The reference-order cell terms run loops whose trip counts follow the
 * cell's set size (pairs and triples of its phases), so lanes of a warp
 * with different sizes idle.  On full-grid launches the kernel walks the
 * cells grouped by set size (each size's cells in grid order within a
 * block); every cell's arithmetic is unchanged. */
struct SetSizeKey {
    const uint16_t *as;
    int P;
    __device__ __forceinline__ int operator()(int64_t c) const
    {
        const int n = as[c];
        return (n >= 1 && n <= P) ? n : 0;
    }
};

template <int DIM, int PM, bool SINGLE>
__global__ void __launch_bounds__(kFp64Block) k_rhs_pf_fp64_ordered(const PfArgs<double> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    CellIndex ci;
    ci.live = t < a.ncells;
    ci.c = ci.live ? (int64_t)a.order[t] : 0;
    ci.x = (int)(ci.c % a.res[0]);
    ci.y = (int)((ci.c / a.res[0]) % a.res[1]);
    ci.z = (int)(ci.c / ((int64_t)a.res[0] * a.res[1]));
    const SlotColumns<double> sc = slot_columns<double>(smem, a.P, blockDim.x, threadIdx.x, true);
    pf_fp64_cell<DIM, PM, SINGLE>(a, ci, sc);
}

/* batched: a persistent grid walks the tiles of every domain of the batch */
template <int DIM, int PM, bool SINGLE, int BY>
__global__ void __launch_bounds__(kBX * BY) k_rhs_pf_fp64_batched(const BatchTiles<double> b)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const SlotColumns<double> sc = slot_columns<double>(smem, b.pmax, blockDim.x, threadIdx.x, true);
    for (int64_t t = blockIdx.x; t < b.total; t += gridDim.x) {
        int inst;
        const CellIndex ci = batch_cell_index<kBX, BY>(b, t, inst);
        if (!b.active[inst]) continue;
        pf_fp64_cell<DIM, PM, SINGLE>(b.args[inst], ci, sc);
    }
}

template <int DIM, int PM>
static void launch_pm(const PfArgs<double> &a, cudaStream_t s)
{
    size_t sm = slot_columns_bytes(a.P, kFp64Block, 8, true);
    const bool whole = a.zcount <= 0 || (a.zbase == 0 && a.zcount >= a.res[2]);
    if (a.order && whole && a.P < kOrderClasses) {
        const OrderBuf o = {a.order, a.order_counts, a.order_cursor, a.P + 1, a.ncells};
        launch_order(o, SetSizeKey{a.as, a.P}, s);
        const unsigned blocks = (unsigned)((a.ncells + kFp64Block - 1) / kFp64Block);
        if (a.single) k_rhs_pf_fp64_ordered<DIM, PM, true><<<blocks, kFp64Block, sm, s>>>(a);
        else k_rhs_pf_fp64_ordered<DIM, PM, false><<<blocks, kFp64Block, sm, s>>>(a);
        return;
    }
    dim3 grid((unsigned)((a.res[0] + kBX - 1) / kBX), (unsigned)((a.res[1] + kBY - 1) / kBY),
              (unsigned)(a.zcount > 0 ? a.zcount : a.res[2]));
    if (a.single) k_rhs_pf_fp64<DIM, PM, true><<<grid, kFp64Block, sm, s>>>(a);
    else k_rhs_pf_fp64<DIM, PM, false><<<grid, kFp64Block, sm, s>>>(a);
}

template <int DIM>
static void launch_dim(const PfArgs<double> &a, cudaStream_t s)
{
    if (a.P <= 4) launch_pm<DIM, 4>(a, s);
    else if (a.P <= 8) launch_pm<DIM, 8>(a, s);
    else if (a.P <= 12) launch_pm<DIM, 12>(a, s);
    else launch_pm<DIM, 16>(a, s);
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

template <int DIM, int PM, bool SINGLE>
static cudaError_t launch_batched_by(const BatchTiles<double> &b, int by, int grid, cudaStream_t s)
{
    const size_t sm = slot_columns_bytes(b.pmax, kBX * by, 8, true);
    cudaError_t e;
    if (by == 1) {
        if ((e = allow_smem(k_rhs_pf_fp64_batched<DIM, PM, SINGLE, 1>, sm)) != cudaSuccess) return e;
        k_rhs_pf_fp64_batched<DIM, PM, SINGLE, 1><<<grid, kBX, sm, s>>>(b);
    } else if (by == 2) {
        if ((e = allow_smem(k_rhs_pf_fp64_batched<DIM, PM, SINGLE, 2>, sm)) != cudaSuccess) return e;
        k_rhs_pf_fp64_batched<DIM, PM, SINGLE, 2><<<grid, kBX * 2, sm, s>>>(b);
    } else {
        if ((e = allow_smem(k_rhs_pf_fp64_batched<DIM, PM, SINGLE, 4>, sm)) != cudaSuccess) return e;
        k_rhs_pf_fp64_batched<DIM, PM, SINGLE, 4><<<grid, kBX * 4, sm, s>>>(b);
    }
    return cudaGetLastError();
}

template <int DIM>
static cudaError_t launch_batched_dim(const BatchTiles<double> &b, int single, int by, int grid, cudaStream_t s)
{
    if (b.pmax <= 4) return single ? launch_batched_by<DIM, 4, true>(b, by, grid, s) : launch_batched_by<DIM, 4, false>(b, by, grid, s);
    if (b.pmax <= 8) return single ? launch_batched_by<DIM, 8, true>(b, by, grid, s) : launch_batched_by<DIM, 8, false>(b, by, grid, s);
    if (b.pmax <= 12) return single ? launch_batched_by<DIM, 12, true>(b, by, grid, s) : launch_batched_by<DIM, 12, false>(b, by, grid, s);
    return single ? launch_batched_by<DIM, 16, true>(b, by, grid, s) : launch_batched_by<DIM, 16, false>(b, by, grid, s);
}

cudaError_t launch_rhs_pf_batched(const BatchTiles<double> &b, int dim, int single, int by, int grid, cudaStream_t s)
{
    if (dim == 1) return launch_batched_dim<1>(b, single, by, grid, s);
    if (dim == 2) return launch_batched_dim<2>(b, single, by, grid, s);
    return launch_batched_dim<3>(b, single, by, grid, s);
}

cudaError_t launch_rhs_phasefield(const PfArgs<double> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_dim<1>(a, s);
    else if (dim == 2) launch_dim<2>(a, s);
    else launch_dim<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
