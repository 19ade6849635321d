/*
 * rhs_items.cu - the model evaluations of the cells of several phases,
 * one thread per (cell, phase) item.
 *
 * For each phase g of a cell of n phases the reference's RHSFunction
 * (src/cipher.c:391-581, 583-662) evaluates the site fractions at the
 * phase's implicit potentials, the chemical energy, the explicit site
 * potentials (dEX/dt) and the site-fraction tangent.  These chains are
 * long (the Redlich-Kister sums of the CALPHAD models) and independent
 * across phases; evaluated one after the other on the cell's thread they
 * make the cells with many phases the tail of the RHS.  Here
 *   k_item_list  : gives each cell of several phases (that the single-phase
 *                  kernels do not take) n consecutive items (a.ibase[c];
 *                  a.icell[item] = cell * 16 + slot); a cell whose items do
 *                  not fit the capacity gets -1 and is evaluated whole by
 *                  the general kernel;
 *   k_items      : per item, the operations the general kernel runs for
 *                  that phase (the interpolant and segregation potential of
 *                  the whole cell, the slot potential, sitefrac, energy,
 *                  explicit potentials, tangent), writing the phase's dEX/dt
 *                  planes of F and its results into the item scratch
 *                  (general_common.cuh: ItemQ), and the phase's mobilities
 *                  for k_chem_cell; the energy, the explicit potentials with
 *                  the tangent, and the mobilities run on three warps.
 * The general kernel then combines each cell's items in the reference's
 * order.  When every material has one model, k_items is compiled for the
 * component count and model (the model bodies inline, models.cuh).
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "general_common.cuh"
#include "kernels.h"
#include "models.cuh"

namespace cipher {

constexpr int kItemBlock = 96;     /* three warps: the three parts of 32 items */

template <typename R>
__global__ void __launch_bounds__(kGenBlock) k_item_list(const GenArgs<R> a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int n = 0;
    if (c < a.ncells) {
        n = a.as[c];
        if (n < 2 || n > a.P || n > CIPHER_PMAX || single_model(a, c) >= 0) n = 0;
    }
    /* warp-aggregated allocation: one atomic per warp */
    int incl = n;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 31 && total) base = atomicAdd(a.icount, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    if (c >= a.ncells) return;
    const int64_t first = (int64_t)base + incl - n;
    if (n && first + n <= a.icap) {
        a.ibase[c] = (int32_t)first;
        for (int g = 0; g < n; g++) a.icell[first + g] = (int32_t)(c * 16 + g);
    } else {
        a.ibase[c] = -1;
        /* a cell whose items straddle the capacity: its entries below it
         * name no item */
        for (int64_t q = first; n && q < first + n && q < a.icap; q++) a.icell[q] = -1;
    }
}

template <int NC, int MODEL, typename R>
__global__ void __launch_bounds__(kItemBlock) k_items(const GenArgs<R> a)
{
    using PMod = PhaseModel<NC, MODEL>;
    const int64_t S = a.stride;
    const int ncp = NC > 0 ? NC : a.ncp, ndp = NC > 0 ? NC - 1 : a.ndp, SP = a.SP;
    const ItemQ iq = item_q(ndp, SP);
    const int64_t nitems = *a.icount < a.icap ? (int64_t)*a.icount : a.icap;
    /* three warps per 32 items: part 0 evaluates the energy (and the
     * site-fraction results), part 1 the explicit potentials and the
     * tangent, part 2 the mobilities (for k_chem_cell), so that the long
     * model chains of an item run side by side; each evaluates the site
     * fractions (the same bits).  The grid stride is a multiple of 96
     * threads, so a thread's part stays the same along the loop. */
    const int64_t nv = 3 * ((nitems + 31) / 32) * 32;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t w = v >> 5;
        const int part = (int)(w % 3);
        const int64_t it = (w / 3) * 32 + (v & 31);
        if (it >= nitems) continue;
        const int32_t code = a.icell[it];
        if (code < 0 || (int64_t)(code >> 4) >= a.ncells) continue;
        const int64_t c = code >> 4;
        const int g = code & 15;
        if (a.ibase[c] != it - g) continue;       /* an entry of an earlier listing */
        uint16_t ids[CIPHER_PMAX];
        double phi[CIPHER_PMAX], h[CIPHER_PMAX];
        const int n = load_set<CIPHER_PMAX>(a, c, ids, phi);
        if (n == 0) continue;
        const double T = (double)a.tm[c];
        const ChemTables ch = chem_at(a.chem, T);
        double mu[CIPHER_MAXCP], ci[CIPHER_MAXCP];
        for (int d = 0; d < ndp; d++) mu[d] = a.dp[(int64_t)d * S + c];
        interpolant(a.interp, phi, n, h);
        segregation<NC>(a, ids, h, n, ci);
        const cipher_material &mat = material_of(ch, ids[g]);
        const int ns = PMod::nsites(mat);
        auto put = [&](int q, double v) { a.iscr[(int64_t)q * a.icap + it] = v; };
        double pot[2 * CIPHER_MAXCP], y[2 * CIPHER_MAXCP];
        slot_potential<NC, MODEL>(a, mat, mu, ci, c, g, pot);
        PMod::sitefrac(ch, ids[g], pot, T, y);
        if (part == 2) {
            /* the phase's share of the cell's composition and mobility
             * (src/cipher.c:148-233) */
            double me[CIPHER_MAXCP];
            PMod::mobility(ch, ids[g], y, T, me);
            for (int d = 0; d < ncp; d++) put(iq.me + d, me[d]);
            for (int s = 0; s < ns; s++)
                for (int d = 0; d < ncp; d++) put(iq.yc + s * ncp + d, y[s * ncp + d]);
            continue;
        }
        if (part == 0) {
            put(0, PMod::chemenergy(ch, ids[g], y, mu, T));
            for (int s = 0; s < ns; s++)
                for (int d = 0; d < ndp; d++) put(iq.y + s * ndp + d, y[s * ncp + d]);
            for (int d = 0; d < ndp; d++) {
                double yw = 0.0;
                for (int s = 0; s < ns; s++) yw += mat.stoichiometry[s] * y[s * ncp + d];
                put(iq.yw + d, yw);
            }
            continue;
        }
        /* explicit potential relaxation (src/cipher.c:570-581) */
        double spx[2 * CIPHER_MAXCP];
        PMod::sitepot_explicit(ch, ids[g], y, T, spx);
        for (int s = 0; s < ns; s++)
            for (int d = 0; d < ndp; d++) {
                const int64_t pl = (int64_t)(g * SP + s * ndp + d) * S + c;
                a.fex[pl] = mat.chempot_ex_kineticcoeff * (spx[s * ndp + d] - a.ex[pl]);
            }
        for (int q = ns * ndp; q < SP; q++) a.fex[(int64_t)(g * SP + q) * S + c] = 0.0;
        double tpot[2 * 16], tex[2 * 16], tT[2 * CIPHER_MAXCP];
        PMod::sitefrac_tangent(ch, ids[g], y, pot, T, tpot, tex, tT);
        for (int q = 0; q < ns * ndp * ndp; q++) {
            put(iq.tpot + q, tpot[q]);
            put(iq.tex + q, tex[q]);
        }
        for (int q = 0; q < ns * ndp; q++) put(iq.tt + q, tT[q]);
    }
}

/* ------------------------------------------------------------------ */
/* launchers                                                            */
/* ------------------------------------------------------------------ */

template <int NC, typename R>
static void launch_items_nc(const GenArgs<R> &a, unsigned grid, cudaStream_t s)
{
    switch (a.item_model) {
    case CIPHER_CHEM_QUADRATIC: k_items<NC, CIPHER_CHEM_QUADRATIC, R><<<grid, kItemBlock, 0, s>>>(a); break;
    case CIPHER_CHEM_CALPHADDIS: k_items<NC, CIPHER_CHEM_CALPHADDIS, R><<<grid, kItemBlock, 0, s>>>(a); break;
    case CIPHER_CHEM_CALPHAD2SL: k_items<NC, CIPHER_CHEM_CALPHAD2SL, R><<<grid, kItemBlock, 0, s>>>(a); break;
    default: k_items<0, -1, R><<<grid, kItemBlock, 0, s>>>(a); break;
    }
}

template <typename R>
static cudaError_t launch_items_t(const GenArgs<R> &a, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(a.icount, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)((a.ncells + kGenBlock - 1) / kGenBlock);
    k_item_list<R><<<blocks, kGenBlock, 0, s>>>(a);
    /* a grid-stride loop over the items listed on the device: a few blocks
     * per SM cover the usual few items per hundred cells in one pass */
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t need = (3 * a.icap + kItemBlock - 1) / kItemBlock;   /* three threads per item */
    const unsigned grid = (unsigned)(need < (int64_t)sms * 16 ? need : (int64_t)sms * 16);
    switch (a.item_model >= 0 ? a.ncp : 0) {
    case 2: launch_items_nc<2>(a, grid, s); break;
    case 3: launch_items_nc<3>(a, grid, s); break;
    case 4: launch_items_nc<4>(a, grid, s); break;
    case 5: launch_items_nc<5>(a, grid, s); break;
    default: k_items<0, -1, R><<<grid, kItemBlock, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_items(const GenArgs<double> &a, cudaStream_t s) { return launch_items_t(a, s); }
cudaError_t launch_items(const GenArgs<float> &a, cudaStream_t s) { return launch_items_t(a, s); }

}  // namespace cipher
