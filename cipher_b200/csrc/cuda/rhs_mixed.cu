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

#ifndef CIPHER_MIXED_BX
#define CIPHER_MIXED_BX 32
#define CIPHER_MIXED_BY 4
#endif

namespace cipher {

constexpr int kBX = CIPHER_MIXED_BX, kBY = CIPHER_MIXED_BY, kMixedBlock = kBX * kBY;

template <int DIM, int PM>
__global__ void __launch_bounds__(kMixedBlock) k_rhs_pf_mixed_single(const PfArgs<float> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const CellIndex ci = cell_index<kBX, kBY>(a.res);
    const SlotColumns<float> sc = slot_columns<float>(smem, a.P, blockDim.x, threadIdx.x, false);
    const int n = load_and_gather<DIM, PM, float, false>(a, ci, sc);
    if (!ci.live) return;
    const int64_t S = a.stride, c = ci.c;
    uint32_t act = 0;
    double nact = 0.0, Ca = 0.0;
    const double mob = a.mob0;
    if (n > 1) {
        const float sig = (float)a.sig0, inv_w = (float)(1.0 / a.wid0);
        const float w_pi2 = (float)(a.wid0 / (CIPHER_PI_D * CIPHER_PI_D));
        const float tjh = (float)(0.5 * a.tj0);
        float A = 0.0f, S1 = 0.0f, S2 = 0.0f;
        for (int k = 0; k < n; k++) {
            const float p = sc.PHI(k);
            A += p * inv_w + sc.LAP(k) * w_pi2;
            S1 += p;
            S2 += p * p;
        }
        /* capillary force, stored over the consumed Laplacian */
        double C = 0.0;
        for (int k = 0; k < n; k++) {
            const float p = sc.PHI(k), l = sc.LAP(k);
            const float ak = p * inv_w + l * w_pi2;
            const float o1 = S1 - p, o2 = S2 - p * p;
            const float cap = 8.0f * (-sig * (A - ak) - tjh * (o1 * o1 - o2)) + l;
            sc.LAP(k) = cap;
            C += (double)cap;
        }
        for (int k = 0; k < n; k++) {
            const double cap = (double)sc.LAP(k);
            const double u = mob * ((double)n * cap - C);
            const double p = (double)sc.PHI(k);
            const bool on = (p > CIPHER_TOL && p < 1.0 - CIPHER_TOL) || (p < CIPHER_TOL && u > 0.0) ||
                            (p > 1.0 - CIPHER_TOL && u < 0.0);
            if (on) { act |= 1u << k; nact += 1.0; Ca += cap; }
        }
    }
    for (int m = 0; m < a.P; m++) {
        float v = 0.0f;
        if (m < n && (act >> m & 1u)) v = (float)(mob * (nact * (double)sc.LAP(m) - Ca) / nact);
        a.fphi[(int64_t)m * S + c] = v;
    }
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = (float)tr;
}

template <int DIM, int PM>
__global__ void __launch_bounds__(kMixedBlock) k_rhs_pf_mixed_multi(const PfArgs<float> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const CellIndex ci = cell_index<kBX, kBY>(a.res);
    const SlotColumns<float> sc = slot_columns<float>(smem, a.P, blockDim.x, threadIdx.x, true);
    const int n = load_and_gather<DIM, PM, float, false>(a, ci, sc);
    const double T = n == 0 ? 0.0 : (double)a.tm[ci.c];
    cell_rates_ordered<float, false>(a, sc, n, ci.c, ci.live, T);
    if (!ci.live) return;
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[ci.c] = (float)tr;
}

template <int DIM, int PM>
static void launch_pm(const PfArgs<float> &a, cudaStream_t s)
{
    dim3 grid((unsigned)((a.res[0] + kBX - 1) / kBX), (unsigned)((a.res[1] + kBY - 1) / kBY), (unsigned)a.res[2]);
    if (a.single) {
        size_t sm = slot_columns_bytes(a.P, kMixedBlock, 4, false);
        k_rhs_pf_mixed_single<DIM, PM><<<grid, kMixedBlock, sm, s>>>(a);
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

cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_dim<1>(a, s);
    else if (dim == 2) launch_dim<2>(a, s);
    else launch_dim<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
