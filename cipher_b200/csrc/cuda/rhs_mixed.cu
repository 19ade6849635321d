/*
 * rhs_mixed.cu - FP32-mixed RHS of the multi-phase-field equation on uniform
 * grids for problems without chemistry (the FP64 version is
 * rhs_phasefield.cu; the equations are src/cipher.c:235-317 and 391-555).
 *
 * Phase fractions, the stencil and the interface terms are FP32 (storage and
 * arithmetic); the pair-rate reductions that decide the active set and the
 * constrained rate are accumulated in FP64.  For a single interface the
 * pair and triple sums of the reference collapse to per-cell sums:
 *   sum_{j != k} sigma*a_j              = sigma*(A - a_k)
 *   sum_{j<i; j,i != k} phi_j*phi_i    = ((S1-phi_k)^2 - (S2-phi_k^2))/2
 *   sum_{j != k} m*(cap_k - cap_j)     = m*(n*cap_k - C)
 * (A = sum a_j, S1 = sum phi_j, S2 = sum phi_j^2, C = sum cap_j), which
 * makes the cell terms O(n) instead of O(n^3).  Several interfaces use the
 * reference-order evaluation of pf_cell.cuh in FP32.  Accuracy against the
 * FP64 oracle on the same inputs: max|dF|/max|F| <= 1e-6 (tested).
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"
#include "pf_cell.cuh"

namespace cipher {

constexpr int kMixedBlock = 128;

template <int DIM, int PM>
__global__ void __launch_bounds__(kMixedBlock) k_rhs_pf_mixed_single(const PfArgs<float> a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = c < a.ncells;
    const int64_t S = a.stride;
    CellPF<PM, float> cp;
    load_and_gather<DIM, PM, float, false>(a, c, live, cp);
    const int n = cp.n;
    float pf[PM];
#pragma unroll
    for (int g = 0; g < PM; g++) pf[g] = 0.0f;

    if (n > 1) {
        const float sig = (float)a.sig0, inv_w = (float)(1.0 / a.wid0);
        const float w_pi2 = (float)(a.wid0 / (CIPHER_PI_D * CIPHER_PI_D));
        const float tjh = (float)(0.5 * a.tj0);
        const double mob = a.mob0;
        float A = 0.0f, S1 = 0.0f, S2 = 0.0f;
#pragma unroll
        for (int k = 0; k < PM; k++)
            if (k < n) {
                A += cp.phi[k] * inv_w + cp.lap[k] * w_pi2;
                S1 += cp.phi[k];
                S2 += cp.phi[k] * cp.phi[k];
            }
        float cap[PM];
        double C = 0.0;
#pragma unroll
        for (int k = 0; k < PM; k++) {
            if (k < n) {
                float ak = cp.phi[k] * inv_w + cp.lap[k] * w_pi2;
                float o1 = S1 - cp.phi[k];
                float o2 = S2 - cp.phi[k] * cp.phi[k];
                cap[k] = 8.0f * (-sig * (A - ak) - tjh * (o1 * o1 - o2)) + cp.lap[k];
                C += (double)cap[k];
            } else {
                cap[k] = 0.0f;
            }
        }
        uint32_t act = 0;
        double nact = 0.0, Ca = 0.0;
#pragma unroll
        for (int k = 0; k < PM; k++) {
            if (k < n) {
                double u = mob * ((double)n * (double)cap[k] - C);
                double p = (double)cp.phi[k];
                bool on = (p > CIPHER_TOL && p < 1.0 - CIPHER_TOL) || (p < CIPHER_TOL && u > 0.0) ||
                          (p > 1.0 - CIPHER_TOL && u < 0.0);
                if (on) { act |= 1u << k; nact += 1.0; Ca += (double)cap[k]; }
            }
        }
#pragma unroll
        for (int k = 0; k < PM; k++)
            if (k < n && (act >> k & 1u)) pf[k] = (float)(mob * (nact * (double)cap[k] - Ca) / nact);
    }
    if (!live) return;
#pragma unroll
    for (int g = 0; g < PM; g++)
        if (g < a.P) a.fphi[(int64_t)g * S + c] = pf[g];
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = (float)tr;
}

template <int DIM, int PM>
__global__ void __launch_bounds__(64) k_rhs_pf_mixed_multi(const PfArgs<float> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = c < a.ncells;
    CellPF<PM, float> cp;
    load_and_gather<DIM, PM, float, false>(a, c, live, cp);
    const int bd = blockDim.x, tid = threadIdx.x;
    float *base = (float *)smem;
    SlotColumns<float> sc;
    sc.st = bd;
    sc.phi = base + tid;
    sc.aj = base + (size_t)PM * bd + tid;
    sc.lap = base + (size_t)2 * PM * bd + tid;
    sc.cap = base + (size_t)3 * PM * bd + tid;
    sc.ids = (uint16_t *)(base + (size_t)4 * PM * bd) + tid;
    const double T = (!live || cp.n == 0) ? 0.0 : (double)a.tm[c];
    cell_rates_ordered<PM, float>(a, cp, sc, c, live, T);
    if (!live) return;
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = (float)tr;
}

template <int DIM, int PM>
static void launch_one(const PfArgs<float> &a, cudaStream_t s)
{
    if (a.single) {
        int64_t blocks = (a.ncells + kMixedBlock - 1) / kMixedBlock;
        k_rhs_pf_mixed_single<DIM, PM><<<(unsigned)blocks, kMixedBlock, 0, s>>>(a);
    } else {
        int64_t blocks = (a.ncells + 63) / 64;
        size_t sm = (size_t)64 * PM * (4 * 4 + 2);
        k_rhs_pf_mixed_multi<DIM, PM><<<(unsigned)blocks, 64, sm, s>>>(a);
    }
}

template <int DIM>
static void launch_pm(const PfArgs<float> &a, cudaStream_t s)
{
    if (a.P <= 4) launch_one<DIM, 4>(a, s);
    else if (a.P <= 8) launch_one<DIM, 8>(a, s);
    else if (a.P <= 12) launch_one<DIM, 12>(a, s);
    else launch_one<DIM, 16>(a, s);
}

cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_pm<1>(a, s);
    else if (dim == 2) launch_pm<2>(a, s);
    else launch_pm<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
