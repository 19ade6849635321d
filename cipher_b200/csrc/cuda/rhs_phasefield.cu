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
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"
#include "pf_cell.cuh"

namespace cipher {

constexpr int kBX = 32, kBY = 2, kFp64Block = kBX * kBY;

template <int DIM, int PM, bool SINGLE>
__global__ void __launch_bounds__(kFp64Block) k_rhs_pf_fp64(const PfArgs<double> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const CellIndex ci = cell_index<kBX, kBY>(a.res);
    const SlotColumns<double> sc = slot_columns<double>(smem, a.P, blockDim.x, threadIdx.x, true);
    const int n = load_and_gather<DIM, PM, double, true>(a, ci, sc);
    const double T = (SINGLE || n == 0) ? 0.0 : a.tm[ci.c];
    cell_rates_ordered<double, SINGLE>(a, sc, n, ci.c, ci.live, T);
    if (!ci.live) return;
    /* temperature: no conductivity, latent or specific heat (src/cipher.c:558-568) */
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[ci.c] = tr;
}

template <int DIM, int PM>
static void launch_pm(const PfArgs<double> &a, cudaStream_t s)
{
    dim3 grid((unsigned)((a.res[0] + kBX - 1) / kBX), (unsigned)((a.res[1] + kBY - 1) / kBY), (unsigned)a.res[2]);
    size_t sm = slot_columns_bytes(a.P, kFp64Block, 8, true);
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

cudaError_t launch_rhs_phasefield(const PfArgs<double> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_dim<1>(a, s);
    else if (dim == 2) launch_dim<2>(a, s);
    else launch_dim<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
