/*
 * ts_vec.cu - vector operations of the time stepper on device states:
 * Y = X + a*F over the PF, DP, EX and TM planes (PETSc's VecAXPY/VecWAXPY
 * on the solution vector; AS entries are exact integers with zero RHS and are
 * copied, as X + a*0 leaves them unchanged).
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "kernels.h"

namespace cipher {

template <typename R>
__global__ void __launch_bounds__(256) k_waxpy(int64_t nreal, int64_t ndbl, const R *xr, const R *fr, R *yr,
                                               const double *xd, const double *fd, double *yd, double a)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = i; k < nreal; k += stride) yr[k] = xr[k] + (R)a * fr[k];
    for (int64_t k = i; k < ndbl; k += stride) yd[k] = xd[k] + a * fd[k];
}

cudaError_t launch_waxpy(int precision, int64_t nreal, int64_t ndbl, const void *xr, const void *fr, void *yr,
                         const double *xd, const double *fd, double *yd, double a, cudaStream_t s)
{
    int64_t n = nreal > ndbl ? nreal : ndbl;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    if (precision == CIPHER_PREC_FP64)
        k_waxpy<double><<<(unsigned)blocks, 256, 0, s>>>(nreal, ndbl, (const double *)xr, (const double *)fr,
                                                          (double *)yr, xd, fd, yd, a);
    else
        k_waxpy<float><<<(unsigned)blocks, 256, 0, s>>>(nreal, ndbl, (const float *)xr, (const float *)fr,
                                                         (float *)yr, xd, fd, yd, a);
    return cudaGetLastError();
}

}  // namespace cipher
