/*
 * rhs_phasefield.cu - FP64 RHS of the multi-phase-field equation on uniform
 * grids for problems without chemistry (every material `none` with a zero
 * reference energy, no segregation potential, D = 0): grain growth.
 *
 * Replaces, for that class of problems, RHSFunction (src/cipher.c:27-681):
 * the face loop (235-317) becomes a per-cell gather over z-marching
 * shared-memory tiles (rhs_tile.cuh) and the cell loop (391-664) runs in the
 * same thread (pf_cell.cuh).
 *
 * Bit-identical to the reference: every value is formed by the same IEEE
 * operations in the same order (this unit is compiled with --fmad=false).
 * All P slots of F are written (zero beyond n).
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"
#include "pf_gather.cuh"
#include "pf_cell.cuh"
#include "rhs_tile.cuh"

namespace cipher {

constexpr int kDX = 32, kDY = 2, kDZC = 8;

template <int DIM, bool SINGLE>
__global__ void __launch_bounds__(kDX * kDY) k_rhs_tile_fp64(const PfArgs<double> a)
{
    using T = TileShape<kDX, kDY>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int P = a.P;
    const size_t pb = tile_plane_bytes<double, T::HC>(P);
    auto plane = [&](int slot) { return tile_plane<double, T::HC>(smem + (size_t)slot * pb, P); };
    double *cb = (double *)(smem + 3 * pb);
    const int tid = threadIdx.x, tx = tid % kDX, ty = tid / kDX;
    SlotColumns<double> sc;
    sc.lap = cb + tid;
    sc.aj = cb + (size_t)P * T::NT + tid;
    sc.cap = cb + (size_t)2 * P * T::NT + tid;
    sc.nz = (uint8_t *)(cb + (size_t)3 * P * T::NT) + tid;
    sc.st = T::NT;
    sc.pst = T::HC;
    const int x0 = blockIdx.x * kDX, y0 = blockIdx.y * kDY, zs = blockIdx.z * kDZC;
    const int ze = min(zs + kDZC, a.res[2]);
    const int gx = x0 + tx, gy = y0 + ty;
    const bool col_live = gx < a.res[0] && gy < a.res[1];
    if (DIM == 3) {
        load_tile_plane<DIM, kDX, kDY, double>(a, plane(0), x0, y0, zs - 1, true);
        load_tile_plane<DIM, kDX, kDY, double>(a, plane(2), x0, y0, zs + 1, true);
    }
    load_tile_plane<DIM, kDX, kDY, double>(a, plane(1), x0, y0, zs, true);
    const int h0 = (ty + 1) * T::HX + tx + 1;
    for (int z = zs; z < ze; z++) {
        const int i = z - zs;
        const TilePlane<double> lo = plane(i % 3), mid = plane((i + 1) % 3), hi = plane((i + 2) % 3);
        __syncthreads();
        if (col_live) {
            const int64_t c = (int64_t)gx + (int64_t)a.res[0] * ((int64_t)gy + (int64_t)a.res[1] * z);
            int n = mid.cnt[h0];
            bool ok = n >= 1 && n <= P;
            for (int g = 0; ok && g < n; g++) ok = mid.ids[g * T::HC + h0] < a.npf;
            if (!ok) {
                atomicOr(a.err, ERR_BADSET);
                for (int m = 0; m < P; m++) a.fphi[(int64_t)m * a.stride + c] = 0.0;
                a.ftm[c] = 0.0;
            } else {
                tile_gather<DIM, kDX, kDY, double, true>(a, lo, mid, hi, tx, ty, gx, gy, z, n, sc.lap, T::NT);
                sc.phi = mid.phi + h0;
                sc.ids = mid.ids + h0;
                const double T0 = SINGLE ? 0.0 : a.tm[c];
                cell_rates_ordered<double, SINGLE>(a, sc, n, c, true, T0);
                /* temperature: no conductivity, latent or specific heat (src/cipher.c:558-568) */
                double tr = 0.0;
                if (a.has_temp_rate) tr += a.temp_rate;
                a.ftm[c] = tr;
            }
        }
        __syncthreads();
        if (DIM == 3 && z + 1 < ze) load_tile_plane<DIM, kDX, kDY, double>(a, plane(i % 3), x0, y0, z + 2, true);
    }
}

template <int DIM, bool SINGLE>
static void launch_tile(const PfArgs<double> &a, cudaStream_t s)
{
    using T = TileShape<kDX, kDY>;
    dim3 grid((unsigned)((a.res[0] + kDX - 1) / kDX), (unsigned)((a.res[1] + kDY - 1) / kDY),
              (unsigned)((a.res[2] + kDZC - 1) / kDZC));
    size_t sm = 3 * tile_plane_bytes<double, T::HC>(a.P) + (size_t)a.P * T::NT * (3 * 8 + 1);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_rhs_tile_fp64<DIM, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set = true;
    }
    k_rhs_tile_fp64<DIM, SINGLE><<<grid, T::NT, sm, s>>>(a);
}

template <int DIM>
static void launch_dim(const PfArgs<double> &a, cudaStream_t s)
{
    if (a.single) launch_tile<DIM, true>(a, s);
    else launch_tile<DIM, false>(a, s);
}

cudaError_t launch_rhs_phasefield(const PfArgs<double> &a, int dim, cudaStream_t s)
{
    if (dim == 1) launch_dim<1>(a, s);
    else if (dim == 2) launch_dim<2>(a, s);
    else launch_dim<3>(a, s);
    return cudaGetLastError();
}

}  // namespace cipher
