/*
 * layout.cu - conversion between the reference's per-cell AoS dof layout
 * (PetscSection of src/cipher.c:1162-1172; offsets src/init.c:1330-1343) and
 * the plane-major device state.  AS entries are rounded to integers the way
 * F2IFUNC does (src/utility.c:24-29).
 *
 * One thread per cell walks its ndof contiguous doubles (the warp's rows are
 * adjacent, so the reads are served from L1 after the first touch) and
 * writes one coalesced element per plane.
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"

namespace cipher {

__global__ void __launch_bounds__(256) k_aos_to_soa(const LayoutArgs a, const double *__restrict__ aos, int64_t c0,
                                                    int64_t c1)
{
    const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    const int64_t S = a.stride;
    const double *row = aos + c * a.ndof;
    for (int k = 0; k <= a.P; k++) {
        double v = row[a.as_off + k];
        double r = round(v);
        a.as[(int64_t)k * S + c] = (r >= 0.0 && r <= 65535.0) ? (uint16_t)r : (uint16_t)0;
    }
    for (int g = 0; g < a.P; g++) {
        double v = row[a.pf_off + g];
        if (a.real_bytes == 8) ((double *)a.phi)[(int64_t)g * S + c] = v;
        else ((float *)a.phi)[(int64_t)g * S + c] = (float)v;
    }
    for (int d = 0; d < a.D; d++) a.dp[(int64_t)d * S + c] = row[a.dp_off + d];
    for (int e = 0; e < a.E; e++) a.ex[(int64_t)e * S + c] = row[a.ex_off + e];
    double t = row[a.tm_off];
    if (a.real_bytes == 8) ((double *)a.tm)[c] = t;
    else ((float *)a.tm)[c] = (float)t;
}

__global__ void __launch_bounds__(256) k_soa_to_aos(const LayoutArgs a, double *__restrict__ aos, int include_as,
                                                    int64_t c0, int64_t c1)
{
    const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    const int64_t S = a.stride;
    double *row = aos + c * a.ndof;
    for (int k = 0; k <= a.P; k++) row[a.as_off + k] = include_as ? (double)a.as[(int64_t)k * S + c] : 0.0;
    for (int g = 0; g < a.P; g++)
        row[a.pf_off + g] = a.real_bytes == 8 ? ((const double *)a.phi)[(int64_t)g * S + c]
                                              : (double)((const float *)a.phi)[(int64_t)g * S + c];
    for (int d = 0; d < a.D; d++) row[a.dp_off + d] = a.dp[(int64_t)d * S + c];
    for (int e = 0; e < a.E; e++) row[a.ex_off + e] = a.ex[(int64_t)e * S + c];
    row[a.tm_off] = a.real_bytes == 8 ? ((const double *)a.tm)[c] : (double)((const float *)a.tm)[c];
}

/* cells [c0, c1) of the domain; aos is the whole domain's AoS array */
cudaError_t launch_aos_to_soa_range(const LayoutArgs &a, const double *aos, int64_t c0, int64_t c1, cudaStream_t s)
{
    if (c1 <= c0) return cudaSuccess;
    const int64_t blocks = (c1 - c0 + 255) / 256;
    k_aos_to_soa<<<(unsigned)blocks, 256, 0, s>>>(a, aos, c0, c1);
    return cudaGetLastError();
}

cudaError_t launch_soa_to_aos_range(const LayoutArgs &a, double *aos, int include_as, int64_t c0, int64_t c1,
                                    cudaStream_t s)
{
    if (c1 <= c0) return cudaSuccess;
    const int64_t blocks = (c1 - c0 + 255) / 256;
    k_soa_to_aos<<<(unsigned)blocks, 256, 0, s>>>(a, aos, include_as, c0, c1);
    return cudaGetLastError();
}

cudaError_t launch_aos_to_soa(const LayoutArgs &a, const double *aos, cudaStream_t s)
{
    return launch_aos_to_soa_range(a, aos, 0, a.ncells, s);
}

cudaError_t launch_soa_to_aos(const LayoutArgs &a, double *aos, int include_as, cudaStream_t s)
{
    return launch_soa_to_aos_range(a, aos, include_as, 0, a.ncells, s);
}

/* SetUpProblem state (src/init.c:1739-1827) from the voxel map: the own
 * phase united with the face neighbours' phases (sorted), phi = 1 for the
 * own phase, T = its material's temperature0, DP and EX zero (the
 * chemistry is filled afterwards).  A set above P raises ERR_CAP and is
 * written truncated. */
__global__ void __launch_bounds__(256) k_init_sharp(const InitArgs a)
{
    const LayoutArgs &L = a.L;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= L.ncells) return;
    const int64_t S = L.stride;
    const int64_t st[3] = {1, (int64_t)a.res[0], (int64_t)a.res[0] * a.res[1]};
    int co[3];
    co[0] = (int)(c % a.res[0]);
    co[1] = (int)((c / a.res[0]) % a.res[1]);
    co[2] = (int)(c / ((int64_t)a.res[0] * a.res[1]));
    const int own = a.voxel[c];
    if (own < 0 || own >= a.npf) {
        atomicOr(a.err, ERR_BADSET);
        return;
    }
    uint16_t set[CIPHER_PMAX + 1];
    int n = 1;
    set[0] = (uint16_t)own;
    bool over = false;
    for (int d = 0; d < a.dim; d++)
        for (int side = 0; side < 2; side++) {
            int64_t nb;
            if (side == 0) nb = co[d] > 0 ? c - st[d] : (a.per[d] ? c + (int64_t)(a.res[d] - 1) * st[d] : -1);
            else nb = co[d] < a.res[d] - 1 ? c + st[d] : (a.per[d] ? c - (int64_t)(a.res[d] - 1) * st[d] : -1);
            if (nb < 0) continue;
            const int v = a.voxel[nb];
            if (v < 0 || v >= a.npf) continue;       /* that cell's own thread flags it */
            int k = 0;
            while (k < n && set[k] < v) k++;
            if (k < n && set[k] == v) continue;
            if (n == L.P) { over = true; continue; }
            for (int m = n; m > k; m--) set[m] = set[m - 1];
            set[k] = (uint16_t)v;
            n++;
        }
    if (over) atomicOr(a.err, ERR_CAP);
    L.as[c] = (uint16_t)n;
    for (int k = 0; k < L.P; k++) {
        L.as[(int64_t)(1 + k) * S + c] = k < n ? set[k] : (uint16_t)0;
        const double v = (k < n && set[k] == own) ? 1.0 : 0.0;
        if (L.real_bytes == 8) ((double *)L.phi)[(int64_t)k * S + c] = v;
        else ((float *)L.phi)[(int64_t)k * S + c] = (float)v;
    }
    for (int d = 0; d < L.D; d++) L.dp[(int64_t)d * S + c] = 0.0;
    for (int q = 0; q < L.E; q++) L.ex[(int64_t)q * S + c] = 0.0;
    if (L.real_bytes == 8) ((double *)L.tm)[c] = a.t0[own];
    else ((float *)L.tm)[c] = (float)a.t0[own];
}

cudaError_t launch_init_sharp(const InitArgs &a, cudaStream_t s)
{
    const int64_t blocks = (a.L.ncells + 255) / 256;
    k_init_sharp<<<(unsigned)blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

/* ------------------------------------------------------------------ */
/* state transfer after a mesh adaptation                               */
/* ------------------------------------------------------------------ */

/* new cell i takes the mean of old cells [src0[i], src0[i] + nsrc[i]): the
 * finite-volume transfer of the forest (children copy their parent, a
 * coarsened family averages into the parent; sums in cell order, then one
 * division, as the host transfer forms them).  The sets are copied from the
 * first old cell (a coarsened family shares its set). */
template <typename R>
__global__ void __launch_bounds__(256) k_transfer(const LayoutArgs dst, const LayoutArgs src, const int64_t *src0,
                                                  const int32_t *nsrc)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dst.ncells) return;
    const int64_t s0 = src0[i];
    const int k = nsrc[i];
    for (int q = 0; q <= dst.P; q++) dst.as[q * dst.stride + i] = src.as[q * src.stride + s0];
    auto mean = [&](auto get) {
        if (k == 1) return get(s0);
        double acc = 0.0;
        for (int j = 0; j < k; j++) acc += get(s0 + j);
        return acc / (double)k;
    };
    const R *sp = (const R *)src.phi;
    R *dp_ = (R *)dst.phi;
    for (int g = 0; g < dst.P; g++)
        dp_[g * dst.stride + i] = (R)mean([&](int64_t c) { return (double)sp[g * src.stride + c]; });
    for (int d = 0; d < dst.D; d++)
        dst.dp[d * dst.stride + i] = mean([&](int64_t c) { return src.dp[d * src.stride + c]; });
    for (int e = 0; e < dst.E; e++)
        dst.ex[e * dst.stride + i] = mean([&](int64_t c) { return src.ex[e * src.stride + c]; });
    const R *st = (const R *)src.tm;
    ((R *)dst.tm)[i] = (R)mean([&](int64_t c) { return (double)st[c]; });
}

cudaError_t launch_transfer(const LayoutArgs &dst, const LayoutArgs &src, const int64_t *src0, const int32_t *nsrc,
                            cudaStream_t s)
{
    if (dst.ncells < 1) return cudaSuccess;
    const unsigned blocks = (unsigned)((dst.ncells + 255) / 256);
    if (dst.real_bytes == 8) k_transfer<double><<<blocks, 256, 0, s>>>(dst, src, src0, nsrc);
    else k_transfer<float><<<blocks, 256, 0, s>>>(dst, src, src0, nsrc);
    return cudaGetLastError();
}

}  // namespace cipher
