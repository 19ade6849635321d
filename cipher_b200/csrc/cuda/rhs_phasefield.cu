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

constexpr int kFp64Block = 64;

template <int PM>
__host__ __device__ constexpr size_t slot_smem_bytes(int block, int rbytes)
{
    return (size_t)block * PM * (4 * rbytes + 2);
}

template <int DIM, int PM>
__global__ void __launch_bounds__(kFp64Block) k_rhs_pf_fp64(const PfArgs<double> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = c < a.ncells;
    CellPF<PM, double> cp;
    load_and_gather<DIM, PM, double, true>(a, c, live, cp);
    const int bd = blockDim.x, tid = threadIdx.x;
    double *base = (double *)smem;
    SlotColumns<double> sc;
    sc.st = bd;
    sc.phi = base + tid;
    sc.aj = base + (size_t)PM * bd + tid;
    sc.lap = base + (size_t)2 * PM * bd + tid;
    sc.cap = base + (size_t)3 * PM * bd + tid;
    sc.ids = (uint16_t *)(base + (size_t)4 * PM * bd) + tid;
    const double T = (a.single || !live || cp.n == 0) ? 0.0 : a.tm[c];
    cell_rates_ordered<PM, double>(a, cp, sc, c, live, T);
    if (!live) return;
    /* temperature: no conductivity, latent or specific heat (src/cipher.c:558-568) */
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = tr;
}

template <int DIM, int PM>
static void launch_one(const PfArgs<double> &a, cudaStream_t s)
{
    int64_t blocks = (a.ncells + kFp64Block - 1) / kFp64Block;
    size_t sm = slot_smem_bytes<PM>(kFp64Block, 8);
    k_rhs_pf_fp64<DIM, PM><<<(unsigned)blocks, kFp64Block, sm, s>>>(a);
}

template <int DIM>
static void launch_pm(const PfArgs<double> &a, cudaStream_t s)
{
    if (a.P <= 4) launch_one<DIM, 4>(a, s);
    else if (a.P <= 8) launch_one<DIM, 8>(a, s);
    else if (a.P <= 12) launch_one<DIM, 12>(a, s);
    else launch_one<DIM, 16>(a, s);
}

cudaError_t launch_rhs_phasefield(const PfArgs<double> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_pm<1>(a, s);
    else if (dim == 2) launch_pm<2>(a, s);
    else launch_pm<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
