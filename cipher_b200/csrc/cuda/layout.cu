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
#include "kernels.h"

namespace cipher {

__global__ void __launch_bounds__(256) k_aos_to_soa(const LayoutArgs a, const double *__restrict__ aos)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
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

__global__ void __launch_bounds__(256) k_soa_to_aos(const LayoutArgs a, double *__restrict__ aos, int include_as)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
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

cudaError_t launch_aos_to_soa(const LayoutArgs &a, const double *aos, cudaStream_t s)
{
    int64_t blocks = (a.ncells + 255) / 256;
    k_aos_to_soa<<<(unsigned)blocks, 256, 0, s>>>(a, aos);
    return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(const LayoutArgs &a, double *aos, int include_as, cudaStream_t s)
{
    int64_t blocks = (a.ncells + 255) / 256;
    k_soa_to_aos<<<(unsigned)blocks, 256, 0, s>>>(a, aos, include_as);
    return cudaGetLastError();
}

}  // namespace cipher
