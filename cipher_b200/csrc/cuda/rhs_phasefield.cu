/*
 * rhs_phasefield.cu - RHS of the multi-phase-field equation on uniform
 * grids for problems without chemistry (every material `none` with a zero
 * reference energy, no segregation potential, D = 0): grain growth.
 *
 * Replaces, for that class of problems, the whole of RHSFunction
 * (src/cipher.c:27-681): the face loop (235-317) becomes a per-cell gather
 * over the 2*dim neighbours, and the cell loop (391-664) runs in the same
 * thread, so the phi-Laplacian never leaves registers/L1.
 *
 * One thread per owned cell.  State planes are read coalesced (x fastest);
 * a warp of 32 consecutive cells reads 32 consecutive ids/phis per plane.
 * Only the planes of active slots (g < n) are read; all P planes of F are
 * written (zeros beyond n), as the reference's F is zero there.
 *
 * Face-flux summation order: the reference adds face contributions in face
 * order, faces being enumerated as (c, c+e_d) by ascending c then d.  For a
 * cell c those are: faces whose L neighbour is below c without wrap (in
 * descending d), then its own faces (ascending d), then the periodic faces
 * whose L neighbour wraps around above c (ascending d).  The kernel sums in
 * exactly that order, so the FP64 path is bit-identical to the reference.
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"

namespace cipher {

template <int PM, typename R>
struct CellSets {
    uint16_t ids[PM];
    R phi[PM];
    R lap[PM];
};

/* one face between this cell and neighbour nb (src/cipher.c:273-288) */
template <int PM, typename R>
__device__ __forceinline__ void face_flux(const PfArgs<R> &a, int n, CellSets<PM, R> &cs,
                                          int64_t nb, bool cell_is_L)
{
    const int64_t S = a.stride;
    int nn = a.as[nb];
    if (nn > a.P) nn = a.P;           /* the neighbour's own thread flags it */
    uint16_t b0 = nn > 0 ? a.as[S + nb] : 0;
    /* the phase flux is gated on the L cell only (src/cipher.c:277) */
    bool gate = cell_is_L ? (n > 1 || cs.ids[0] > 1) : (nn > 1 || b0 > 1);
    if (!gate) return;
    const R ff = (R)a.ffactor, vol = (R)a.vol;
    int i = 0, j = 0;
    uint16_t b = b0;
    while (i < n && j < nn) {
        uint16_t v = cs.ids[i];
        if (v == b) {
            R pn = a.phi[(int64_t)j * S + nb];
            if (cell_is_L) {
                R flux = pn - cs.phi[i];
                cs.lap[i] += ff * flux / vol;
            } else {
                R flux = cs.phi[i] - pn;
                cs.lap[i] -= ff * flux / vol;
            }
            i++;
            j++;
            if (j < nn) b = a.as[(int64_t)(1 + j) * S + nb];
        } else if (v < b) {
            i++;
        } else {
            j++;
            if (j < nn) b = a.as[(int64_t)(1 + j) * S + nb];
        }
    }
}

template <int DIM, int PM, typename R>
__global__ void __launch_bounds__(256) k_rhs_phasefield(const PfArgs<R> a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    const int64_t S = a.stride;
    int n = a.as[c];
    if (n < 1 || n > a.P) {
        atomicOr(a.err, ERR_BADSET);
        for (int g = 0; g < a.P; g++) a.fphi[(int64_t)g * S + c] = (R)0;
        a.ftm[c] = (R)0;
        return;
    }
    CellSets<PM, R> cs;
    bool badid = false;
#pragma unroll
    for (int g = 0; g < PM; g++) {
        if (g < n) {
            cs.ids[g] = a.as[(int64_t)(1 + g) * S + c];
            cs.phi[g] = a.phi[(int64_t)g * S + c];
            cs.lap[g] = (R)0;
            badid |= cs.ids[g] >= a.npf;
        }
    }
    if (badid) {   /* ids index the interface table: never read past it */
        atomicOr(a.err, ERR_BADSET);
        for (int g = 0; g < a.P; g++) a.fphi[(int64_t)g * S + c] = (R)0;
        a.ftm[c] = (R)0;
        return;
    }

    /* neighbours in the reference's face order */
    const int res[3] = {a.res[0], a.res[1], a.res[2]};
    const int64_t st[3] = {1, (int64_t)res[0], (int64_t)res[0] * res[1]};
    int co[3];
    co[0] = (int)(c % res[0]);
    co[1] = DIM > 1 ? (int)((c / res[0]) % res[1]) : 0;
    co[2] = DIM > 2 ? (int)(c / ((int64_t)res[0] * res[1])) : 0;
#pragma unroll
    for (int d = DIM - 1; d >= 0; d--)
        if (co[d] > 0) face_flux<PM, R>(a, n, cs, c - st[d], false);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        if (co[d] < res[d] - 1) face_flux<PM, R>(a, n, cs, c + st[d], true);
        else if (a.per[d]) face_flux<PM, R>(a, n, cs, c - (int64_t)(res[d] - 1) * st[d], true);
    }
#pragma unroll
    for (int d = 0; d < DIM; d++)
        if (co[d] == 0 && a.per[d]) face_flux<PM, R>(a, n, cs, c + (int64_t)(res[d] - 1) * st[d], false);

    /* cell terms (src/cipher.c:417-555) */
    R pf[PM];
#pragma unroll
    for (int g = 0; g < PM; g++) pf[g] = (R)0;
    if (n > 1) {
        const R PI = (R)CIPHER_PI_D;
        R cap[PM];
        double T = a.single ? 0.0 : (double)a.tm[c];
#pragma unroll
        for (int g = 0; g < PM; g++) cap[g] = (R)0;
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                R sig, wid;
                if (a.single) {
                    sig = (R)a.sig0;
                    wid = (R)a.wid0;
                } else {
                    double s, m, w;
                    interface_props(a.itfs[a.itflist[(int)cs.ids[k] * a.npf + cs.ids[j]]], T, s, m, w);
                    sig = (R)s;
                    wid = (R)w;
                }
                cap[k] -= sig * (cs.phi[j] / wid + cs.lap[j] * wid / PI / PI);
                cap[j] -= sig * (cs.phi[k] / wid + cs.lap[k] * wid / PI / PI);
                for (int i = j + 1; i < n; i++) {
                    R tj;
                    if (a.single) {
                        tj = (R)a.tj0;
                    } else {
                        double s, m, w, v, t = 0.0;
                        interface_props(a.itfs[a.itflist[(int)cs.ids[k] * a.npf + cs.ids[j]]], T, s, m, w);
                        v = s / w; t = t > v ? t : v;
                        interface_props(a.itfs[a.itflist[(int)cs.ids[k] * a.npf + cs.ids[i]]], T, s, m, w);
                        v = s / w; t = t > v ? t : v;
                        interface_props(a.itfs[a.itflist[(int)cs.ids[j] * a.npf + cs.ids[i]]], T, s, m, w);
                        v = s / w; t = t > v ? t : v;
                        t *= a.junctionpenalty;
                        tj = (R)t;
                    }
                    cap[k] -= tj * cs.phi[j] * cs.phi[i];
                    cap[j] -= tj * cs.phi[k] * cs.phi[i];
                    cap[i] -= tj * cs.phi[k] * cs.phi[j];
                }
            }
            cap[k] *= (R)8.0;
            cap[k] += cs.lap[k];
        }
        /* no chemistry: the chemical term is identically zero, so the pair
         * rate is m*(cap_k - cap_j) exactly (src/cipher.c:530-532) */
        R unc[PM];
#pragma unroll
        for (int g = 0; g < PM; g++) unc[g] = (R)0;
        uint32_t act = 0;
        double nact = 0.0;
        for (int k = 0; k < n; k++) {
            for (int j = k + 1; j < n; j++) {
                R mob;
                if (a.single) mob = (R)a.mob0;
                else {
                    double s, m, w;
                    interface_props(a.itfs[a.itflist[(int)cs.ids[k] * a.npf + cs.ids[j]]], T, s, m, w);
                    mob = (R)m;
                }
                R r = mob * (cap[k] - cap[j]);
                unc[k] += r;
                unc[j] -= r;
            }
            double p = (double)cs.phi[k];
            bool on = (p > CIPHER_TOL && p < 1.0 - CIPHER_TOL)
                   || (p < CIPHER_TOL && unc[k] > (R)0)
                   || (p > 1.0 - CIPHER_TOL && unc[k] < (R)0);
            if (on) { act |= 1u << k; nact += 1.0; }
        }
        for (int k = 0; k < n; k++) {
            if (!(act >> k & 1u)) continue;
            for (int j = k + 1; j < n; j++) {
                if (!(act >> j & 1u)) continue;
                R mob;
                if (a.single) mob = (R)a.mob0;
                else {
                    double s, m, w;
                    interface_props(a.itfs[a.itflist[(int)cs.ids[k] * a.npf + cs.ids[j]]], T, s, m, w);
                    mob = (R)m;
                }
                R r = mob * (cap[k] - cap[j]);
                pf[k] += r;
                pf[j] -= r;
            }
            pf[k] /= (R)nact;
        }
    }
#pragma unroll
    for (int g = 0; g < PM; g++)
        if (g < a.P) a.fphi[(int64_t)g * S + c] = g < n ? pf[g] : (R)0;
    /* temperature: no conductivity, latent or specific heat here (src/cipher.c:558-568) */
    double tr = 0.0;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = (R)tr;
}

template <typename R>
static cudaError_t launch_dim(const PfArgs<R> &a, int dim, cudaStream_t s)
{
    int64_t blocks = (a.ncells + 255) / 256;
    dim3 grid((unsigned)blocks), block(256);
    int pm = a.P <= 4 ? 4 : a.P <= 8 ? 8 : a.P <= 12 ? 12 : 16;
#define CIPHER_LAUNCH(D, PMV) k_rhs_phasefield<D, PMV, R><<<grid, block, 0, s>>>(a)
    if (dim == 2) {
        if (pm == 4) CIPHER_LAUNCH(2, 4);
        else if (pm == 8) CIPHER_LAUNCH(2, 8);
        else if (pm == 12) CIPHER_LAUNCH(2, 12);
        else CIPHER_LAUNCH(2, 16);
    } else if (dim == 3) {
        if (pm == 4) CIPHER_LAUNCH(3, 4);
        else if (pm == 8) CIPHER_LAUNCH(3, 8);
        else if (pm == 12) CIPHER_LAUNCH(3, 12);
        else CIPHER_LAUNCH(3, 16);
    } else {
        if (pm == 4) CIPHER_LAUNCH(1, 4);
        else if (pm == 8) CIPHER_LAUNCH(1, 8);
        else if (pm == 12) CIPHER_LAUNCH(1, 12);
        else CIPHER_LAUNCH(1, 16);
    }
#undef CIPHER_LAUNCH
    return cudaGetLastError();
}

cudaError_t launch_rhs_phasefield(const PfArgs<double> &a, int dim, cudaStream_t s) { return launch_dim(a, dim, s); }
cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s) { return launch_dim(a, dim, s); }

}  // namespace cipher
