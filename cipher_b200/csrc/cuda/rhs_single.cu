/*
 * rhs_single.cu - the general RHS for cells that hold a single phase, one
 * kernel per component count and chemical model.
 *
 * In alloy microstructures most cells lie inside a grain or precipitate
 * and hold one phase.  For such a cell the reference's RHSFunction
 * (src/cipher.c:27-681) reduces to: site fractions, mobility and
 * composition of the one phase (148-233), the chemical-potential and heat
 * fluxes of its faces (235-317) and boundary faces (319-389), and the cell
 * terms with h = 1 (or phi with the linear interpolant) and no pairs: a
 * zero phase rate, dT/dt, the explicit-potential relaxation dEX/dt and the
 * composition rate through the inverted tangent dmu/dc (558-662).
 *
 * The kernels here run exactly those operations, in the same order, as the
 * general kernels (rhs_general.cu) run for the same cell, so the results
 * are the same bits; the general kernels skip these cells.  What differs is
 * the code: the component count NC and the model are template arguments,
 * the model bodies (models.cuh) are inlined with their loops unrolled, and
 * every per-component array stays in registers instead of the general
 * kernel's per-thread stack.
 *   k_chem_single : composition, mobility and conductivity planes (the
 *                   neighbours' face fluxes read them);
 *   k_rhs_single  : F of the cell.
 * Both walk the cell grouping (order.cuh), in which the single-phase cells
 * of one material are contiguous runs; a thread whose cell is not of the
 * kernel's model returns at once.
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "general_common.cuh"
#include "kernels.h"
#include "models.cuh"

namespace cipher {

template <int NC, int MODEL, typename R>
__global__ void __launch_bounds__(kGenBlock, 3) k_chem_single(const GenArgs<R> a)
{
    constexpr int ND = NC - 1, NS = model_nsites(MODEL);
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ncells) return;
    const int64_t c = a.order ? (int64_t)a.order[t] : t;
    if (single_model(a, c) != MODEL) return;
    const int64_t S = a.stride;
    const int id = a.as[S + c];
    const double phi0 = (double)a.phi[c];
    const double T = (double)a.tm[c];
    const ChemTables ch = chem_at(a.chem, T);
    const cipher_material &mat = material_of(ch, id);
    /* interpolant of a one-phase set (src/utility.c:470-500) */
    const double h0 = a.interp == CIPHER_INTERP_LINEAR ? phi0 : 1.0;
    double pot[2 * ND], y[2 * NC];
    /* slot potentials with a zero segregation potential */
#pragma unroll
    for (int s = 0; s < NS; s++) {
#pragma unroll
        for (int d = 0; d < ND; d++)
            pot[s * ND + d] = mat.stoichiometry[s] * (a.dp[(int64_t)d * S + c] - 0.0) - a.ex[(int64_t)(s * ND + d) * S + c];
    }
    PhaseModel<NC, MODEL>::sitefrac(ch, id, pot, T, y);
    double me[NC];
    PhaseModel<NC, MODEL>::mobility(ch, id, y, T, me);
#pragma unroll
    for (int d = 0; d < NC; d++) {
        double cc = 0.0;
#pragma unroll
        for (int s = 0; s < NS; s++) cc += h0 * mat.stoichiometry[s] * y[s * NC + d];
        a.comp[(int64_t)d * S + c] = cc;
        a.mob[(int64_t)d * S + c] = 0.0 + h0 * me[d];
    }
    double tc = 0.0;
    if (mat.tconductivity.n) tc += h0 * tseries(T, mat.tconductivity);
    a.tcond[c] = tc;
}

template <int NC, int MODEL, typename R>
__global__ void __launch_bounds__(kGenBlock, 5) k_rhs_single(const GenArgs<R> a, const int DIM)
{
    constexpr int ND = NC - 1, NS = model_nsites(MODEL);
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ncells) return;
    const int64_t c = a.order ? (int64_t)a.order[t] : t;
    if (single_model(a, c) != MODEL) return;
    const int64_t S = a.stride;
    const int SP = a.SP;
    const int id = a.as[S + c];
    const double phi0 = (double)a.phi[c];
    const double T = (double)a.tm[c];
    const ChemTables ch = chem_at(a.chem, T);
    const cipher_material &mat = material_of(ch, id);
    int co[3] = {0, 0, 0};
    if (!a.fl.start) {
        co[0] = (int)(c % a.res[0]);
        co[1] = DIM > 1 ? (int)((c / a.res[0]) % a.res[1]) : 0;
        co[2] = DIM > 2 ? (int)(c / ((int64_t)a.res[0] * a.res[1])) : 0;
    }
    double mu[ND], ldp[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) { mu[d] = a.dp[(int64_t)d * S + c]; ldp[d] = 0.0; }
    double ltm = 0.0;

    /* faces: the chemical-potential and heat fluxes (the phase flux feeds
     * only the pair terms, which a one-phase cell has none of) */
    walk_faces(a, c, co, DIM, [&](int64_t nb, bool self_L, int, const auto &fdiv) {
        const int64_t cl = self_L ? c : nb, cr = self_L ? nb : c;
        chem_heat_face<NC>(a, cl, cr, self_L, fdiv, ldp, ltm);
    });
    boundary_faces<NC>(a, c, co, DIM, T, mu, ldp, ltm);

    /* cell terms (src/cipher.c:391-664) with one phase */
    const double h0 = a.interp == CIPHER_INTERP_LINEAR ? phi0 : 1.0;
    for (int g = 0; g < a.P; g++) a.fphi[(int64_t)g * S + c] = (R)0.0;

    /* temperature rate (src/cipher.c:558-568); the phase rate is zero */
    double cp = 0.0, tr = ltm;
    if (mat.specific_heat.n) cp += h0 * tseries(T, mat.specific_heat);
    if (mat.latent_heat.n) tr += 0.0 * tseries(T, mat.latent_heat);
    if (cp != 0.0) tr /= cp;
    if (a.has_temp_rate) tr += a.temp_rate;
    a.ftm[c] = (R)tr;

    /* solute sources (material.c:295-351) */
    double wdp[ND];
    {
        double src[NC], comp[NC];
#pragma unroll
        for (int d = 0; d < NC; d++) { src[d] = 0.0; comp[d] = a.comp[(int64_t)d * S + c]; }
        for (int s = 0; s < mat.nsources; s++) {
            double tmp[NC];
#pragma unroll
            for (int d = 0; d < NC; d++) tmp[d] = mat.sources[s].rate[d] * (mat.sources[s].ceq[d] - comp[d]);
#pragma unroll
            for (int d = 0; d < NC; d++) src[d] += h0 * h0 * tmp[d];
        }
#pragma unroll
        for (int d = 0; d < ND; d++) wdp[d] = 0.0 + (ldp[d] + src[d]);
    }

    /* site fractions, explicit-potential relaxation, tangent */
    double pot[2 * ND], y[2 * NC];
#pragma unroll
    for (int s = 0; s < NS; s++) {
#pragma unroll
        for (int d = 0; d < ND; d++)
            pot[s * ND + d] = mat.stoichiometry[s] * (mu[d] - 0.0) - a.ex[(int64_t)(s * ND + d) * S + c];
    }
    PhaseModel<NC, MODEL>::sitefrac(ch, id, pot, T, y);
    double fex[2 * ND];
    {
        double spx[2 * ND];
        PhaseModel<NC, MODEL>::sitepot_explicit(ch, id, y, T, spx);
#pragma unroll
        for (int s = 0; s < NS; s++) {
#pragma unroll
            for (int d = 0; d < ND; d++) {
                const int64_t pl = (int64_t)(s * ND + d) * S + c;
                fex[s * ND + d] = mat.chempot_ex_kineticcoeff * (spx[s * ND + d] - a.ex[pl]);
                a.fex[pl] = fex[s * ND + d];
            }
        }
    }
    for (int q = NS * ND; q < a.P * SP; q++) a.fex[(int64_t)q * S + c] = 0.0;
    double tpot[2 * ND * ND], tex[2 * ND * ND], tT[2 * ND];
    PhaseModel<NC, MODEL>::sitefrac_tangent(ch, id, y, pot, T, tpot, tex, tT);
    double dcdm[ND * ND];
#pragma unroll
    for (int q = 0; q < ND * ND; q++) dcdm[q] = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
#pragma unroll
        for (int q = 0; q < ND * ND; q++) dcdm[q] += h0 * mat.stoichiometry[s] * mat.stoichiometry[s] * tpot[s * ND * ND + q];
    }

    /* composition rate and dmu/dt (src/cipher.c:583-662): no pair
     * potentials, so the phase's potential correction is dcdm * 0 */
    double cpv[ND];
    {
        double zero[ND];
#pragma unroll
        for (int d = 0; d < ND; d++) zero[d] = 0.0;
        matvec(cpv, dcdm, zero, ND);
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        matvec(cpv, &tex[s * ND * ND], &fex[s * ND], ND);
#pragma unroll
        for (int d = 0; d < ND; d++) wdp[d] -= h0 * mat.stoichiometry[s] * (cpv[d] + tT[s * ND + d] * tr);
    }
    double dmdc[ND * ND], out[ND];
    invert_small(dmdc, dcdm, ND);
    matvec(out, dmdc, wdp, ND);
#pragma unroll
    for (int d = 0; d < ND; d++) a.fdp[(int64_t)d * S + c] = out[d];
}

/* ------------------------------------------------------------------ */
/* launchers: one launch per model present                              */
/* ------------------------------------------------------------------ */

template <int NC, typename R>
static void launch_models(const GenArgs<R> &a, int dim, bool rhs, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((a.ncells + kGenBlock - 1) / kGenBlock);
    const uint32_t m = a.single_models;
    if (rhs) {
        if (m >> CIPHER_CHEM_NONE & 1u) k_rhs_single<NC, CIPHER_CHEM_NONE, R><<<blocks, kGenBlock, 0, s>>>(a, dim);
        if (m >> CIPHER_CHEM_QUADRATIC & 1u) k_rhs_single<NC, CIPHER_CHEM_QUADRATIC, R><<<blocks, kGenBlock, 0, s>>>(a, dim);
        if (m >> CIPHER_CHEM_CALPHADDIS & 1u) k_rhs_single<NC, CIPHER_CHEM_CALPHADDIS, R><<<blocks, kGenBlock, 0, s>>>(a, dim);
        if (m >> CIPHER_CHEM_CALPHAD2SL & 1u) k_rhs_single<NC, CIPHER_CHEM_CALPHAD2SL, R><<<blocks, kGenBlock, 0, s>>>(a, dim);
    } else {
        if (m >> CIPHER_CHEM_NONE & 1u) k_chem_single<NC, CIPHER_CHEM_NONE, R><<<blocks, kGenBlock, 0, s>>>(a);
        if (m >> CIPHER_CHEM_QUADRATIC & 1u) k_chem_single<NC, CIPHER_CHEM_QUADRATIC, R><<<blocks, kGenBlock, 0, s>>>(a);
        if (m >> CIPHER_CHEM_CALPHADDIS & 1u) k_chem_single<NC, CIPHER_CHEM_CALPHADDIS, R><<<blocks, kGenBlock, 0, s>>>(a);
        if (m >> CIPHER_CHEM_CALPHAD2SL & 1u) k_chem_single<NC, CIPHER_CHEM_CALPHAD2SL, R><<<blocks, kGenBlock, 0, s>>>(a);
    }
}

template <typename R>
static cudaError_t launch_single(const GenArgs<R> &a, int dim, bool rhs, cudaStream_t s)
{
    switch (a.ncp) {
    case 2: launch_models<2>(a, dim, rhs, s); break;
    case 3: launch_models<3>(a, dim, rhs, s); break;
    case 4: launch_models<4>(a, dim, rhs, s); break;
    case 5: launch_models<5>(a, dim, rhs, s); break;
    default: return cudaErrorInvalidValue;      /* the host enables these kernels for 2 <= ncp <= 5 only */
    }
    return cudaGetLastError();
}

cudaError_t launch_chem_single(const GenArgs<double> &a, cudaStream_t s) { return launch_single(a, 0, false, s); }
cudaError_t launch_chem_single(const GenArgs<float> &a, cudaStream_t s) { return launch_single(a, 0, false, s); }
cudaError_t launch_rhs_single(const GenArgs<double> &a, int dim, cudaStream_t s) { return launch_single(a, dim, true, s); }
cudaError_t launch_rhs_single(const GenArgs<float> &a, int dim, cudaStream_t s) { return launch_single(a, dim, true, s); }

}  // namespace cipher
