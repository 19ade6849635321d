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
 *
 * Data movement: z-marching shared-memory tiles (rhs_tile.cuh).
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"
#include "pf_cell.cuh"
#include "rhs_tile.cuh"

namespace cipher {

constexpr int kMX = 32, kMY = 4, kMZC = 8;

/* closed-form cell terms for one interface; writes all P slots of F */
__device__ __forceinline__ void mixed_single_cell(const PfArgs<float> &a, const TilePlane<float> &mid, int HC, int h0,
                                                  int n, const float *lap, int lst, int64_t c)
{
    const int64_t S = a.stride;
    uint32_t act = 0;
    double nact = 0.0, Ca = 0.0;
    const double mob = a.mob0;
    float cap[CIPHER_PMAX];
    if (n > 1) {
        const float sig = (float)a.sig0, inv_w = (float)(1.0 / a.wid0);
        const float w_pi2 = (float)(a.wid0 / (CIPHER_PI_D * CIPHER_PI_D));
        const float tjh = (float)(0.5 * a.tj0);
        float A = 0.0f, S1 = 0.0f, S2 = 0.0f;
        for (int k = 0; k < n; k++) {
            const float p = mid.phi[k * HC + h0];
            A += p * inv_w + lap[k * lst] * w_pi2;
            S1 += p;
            S2 += p * p;
        }
        double C = 0.0;
#pragma unroll
        for (int k = 0; k < CIPHER_PMAX; k++) {
            if (k < n) {
                const float p = mid.phi[k * HC + h0], l = lap[k * lst];
                const float ak = p * inv_w + l * w_pi2;
                const float o1 = S1 - p, o2 = S2 - p * p;
                cap[k] = 8.0f * (-sig * (A - ak) - tjh * (o1 * o1 - o2)) + l;
                C += (double)cap[k];
            }
        }
#pragma unroll
        for (int k = 0; k < CIPHER_PMAX; k++) {
            if (k < n) {
                const double u = mob * ((double)n * (double)cap[k] - C);
                const double p = (double)mid.phi[k * HC + h0];
                const bool on = (p > CIPHER_TOL && p < 1.0 - CIPHER_TOL) || (p < CIPHER_TOL && u > 0.0) ||
                                (p > 1.0 - CIPHER_TOL && u < 0.0);
                if (on) { act |= 1u << k; nact += 1.0; Ca += (double)cap[k]; }
            }
        }
    }
#pragma unroll
    for (int m = 0; m < CIPHER_PMAX; m++) {
        if (m >= a.P) break;
        float v = 0.0f;
        if (m < n && (act >> m & 1u)) v = (float)(mob * (nact * (double)cap[m] - Ca) / nact);
        a.fphi[(int64_t)m * S + c] = v;
    }
}

template <int DIM, bool SINGLE>
__global__ void __launch_bounds__(kMX * kMY) k_rhs_tile_mixed(const PfArgs<float> a)
{
    using T = TileShape<kMX, kMY>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int P = a.P;
    const size_t pb = tile_plane_bytes<float, T::HC>(P);
    auto plane = [&](int slot) { return tile_plane<float, T::HC>(smem + (size_t)slot * pb, P); };
    unsigned char *cols = smem + 3 * pb;
    const int tid = threadIdx.x, tx = tid % kMX, ty = tid / kMX;
    const int x0 = blockIdx.x * kMX, y0 = blockIdx.y * kMY, zs = blockIdx.z * kMZC;
    const int ze = min(zs + kMZC, a.res[2]);
    const int gx = x0 + tx, gy = y0 + ty;
    const bool col_live = gx < a.res[0] && gy < a.res[1];
    /* private columns: lap [P][NT] (+ aj, cap [P][NT], nz for several interfaces) */
    float *lap = (float *)cols + tid;
    SlotColumns<float> sc;
    if (!SINGLE) {
        float *fb = (float *)cols;
        sc.lap = fb + tid;
        sc.aj = fb + (size_t)P * T::NT + tid;
        sc.cap = fb + (size_t)2 * P * T::NT + tid;
        sc.nz = (uint8_t *)(fb + (size_t)3 * P * T::NT) + tid;
        sc.st = T::NT;
        sc.pst = T::HC;
    }
    if (DIM == 3) {
        load_tile_plane<DIM, kMX, kMY, float>(a, plane(0), x0, y0, zs - 1, true);
        load_tile_plane<DIM, kMX, kMY, float>(a, plane(2), x0, y0, zs + 1, zs + 1 < a.res[2] || a.per[2]);
    }
    load_tile_plane<DIM, kMX, kMY, float>(a, plane(1), x0, y0, zs, true);
    const int h0 = (ty + 1) * T::HX + tx + 1;
    for (int z = zs; z < ze; z++) {
        const int i = z - zs;
        const TilePlane<float> lo = plane(i % 3), mid = plane((i + 1) % 3), hi = plane((i + 2) % 3);
        __syncthreads();
        if (col_live) {
            const int64_t c = (int64_t)gx + (int64_t)a.res[0] * ((int64_t)gy + (int64_t)a.res[1] * z);
            int n = mid.cnt[h0];
            bool ok = n >= 1 && n <= P;
            for (int g = 0; ok && g < n; g++) ok = mid.ids[g * T::HC + h0] < a.npf;
            if (!ok) {
                atomicOr(a.err, ERR_BADSET);
                for (int m = 0; m < P; m++) a.fphi[(int64_t)m * a.stride + c] = 0.0f;
                a.ftm[c] = 0.0f;
            } else {
                if (SINGLE) {
                    tile_gather<DIM, kMX, kMY, float, false>(a, lo, mid, hi, tx, ty, gx, gy, z, n, lap, T::NT);
                    mixed_single_cell(a, mid, T::HC, h0, n, lap, T::NT, c);
                } else {
                    tile_gather<DIM, kMX, kMY, float, false>(a, lo, mid, hi, tx, ty, gx, gy, z, n, sc.lap, T::NT);
                    sc.phi = mid.phi + h0;
                    sc.ids = mid.ids + h0;
                    cell_rates_ordered<float, false>(a, sc, n, c, true, (double)a.tm[c]);
                }
                double tr = 0.0;
                if (a.has_temp_rate) tr += a.temp_rate;
                a.ftm[c] = (float)tr;
            }
        }
        __syncthreads();
        if (DIM == 3 && z + 1 < ze) {
            const int zn = z + 2;
            load_tile_plane<DIM, kMX, kMY, float>(a, plane(i % 3), x0, y0, zn, zn < a.res[2] || a.per[2]);
        }
    }
}

template <int DIM, bool SINGLE>
static void launch_tile(const PfArgs<float> &a, cudaStream_t s)
{
    using T = TileShape<kMX, kMY>;
    dim3 grid((unsigned)((a.res[0] + kMX - 1) / kMX), (unsigned)((a.res[1] + kMY - 1) / kMY),
              (unsigned)((a.res[2] + kMZC - 1) / kMZC));
    size_t cols = SINGLE ? (size_t)a.P * T::NT * 4 : (size_t)a.P * T::NT * (3 * 4 + 1);
    size_t sm = 3 * tile_plane_bytes<float, T::HC>(a.P) + cols;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_rhs_tile_mixed<DIM, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set = true;
    }
    k_rhs_tile_mixed<DIM, SINGLE><<<grid, T::NT, sm, s>>>(a);
}

template <int DIM>
static void launch_dim(const PfArgs<float> &a, cudaStream_t s)
{
    if (a.single) launch_tile<DIM, true>(a, s);
    else launch_tile<DIM, false>(a, s);
}

cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_dim<1>(a, s);
    else if (dim == 2) launch_dim<2>(a, s);
    else launch_dim<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
