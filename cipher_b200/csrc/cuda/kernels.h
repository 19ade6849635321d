/*
 * kernels.h - launch interfaces of the device kernels (internal to the
 * library; the public C ABI is include/cipher_b200.h).
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "device_common.cuh"

namespace cipher {

/* arguments of the phase-field-only RHS on a uniform grid */
template <typename R>
struct PfArgs {
    int64_t ncells, stride;
    int res[3];
    int per[3];
    int P, npf;
    double ffactor, vol;          /* face factor and cell volume (src/cipher.c:273-275) */
    int geom_mode;                /* GEOM_DIVIDE / GEOM_RECIP / GEOM_UNIT (pf_gather.cuh) */
    double inv_vol;               /* 1/vol, exact when vol is a power of two */
    double face_coef;             /* ffactor/vol, for the mixed path */
    double junctionpenalty;
    int has_temp_rate;
    double temp_rate;
    int single;                   /* every pair uses one T-independent interface */
    double sig0, mob0, wid0, tj0; /* its sigma, m, w and triple-junction weight */
    const int32_t *itflist;
    const DevInterface *itfs;
    const uint16_t *as;
    const R *phi;
    const R *tm;
    R *fphi;
    R *ftm;
    int *err;
};

cudaError_t launch_rhs_phasefield(const PfArgs<double> &a, int dim, cudaStream_t s);
cudaError_t launch_rhs_phasefield(const PfArgs<float> &a, int dim, cudaStream_t s);

/* per-step active-set update on a uniform grid (src/cipher.c:869-974) */
template <typename R>
struct PostArgs {
    int64_t ncells, stride;
    int res[3];
    int per[3];
    int P, S;                     /* S = explicit site potentials per phase */
    uint16_t *as;
    R *phi;
    double *ex;
    const R *tm;
    uint16_t *pruned;             /* scratch: pruned sets, [P+1][stride] */
    const double *ex_init;        /* [npf*S] explicit potential of c0 at T0 per phase, or NULL */
    int *err;
};

cudaError_t launch_poststep(const PostArgs<double> &a, int dim, cudaStream_t s);
cudaError_t launch_poststep(const PostArgs<float> &a, int dim, cudaStream_t s);

/* reference AoS (ncells x ndof doubles) <-> plane-major device state */
struct LayoutArgs {
    int64_t ncells, stride;
    int P, D, E;                  /* PF slots, DP count, EX count (P*S) */
    int ndof, as_off, pf_off, dp_off, ex_off, tm_off;
    int real_bytes;               /* 8 (FP64) or 4 (mixed) for PF and TM */
    uint16_t *as;
    void *phi;
    double *dp;
    double *ex;
    void *tm;
};
cudaError_t launch_aos_to_soa(const LayoutArgs &a, const double *aos, cudaStream_t s);
cudaError_t launch_soa_to_aos(const LayoutArgs &a, double *aos, int include_as, cudaStream_t s);

}  // namespace cipher
