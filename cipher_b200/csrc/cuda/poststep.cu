/*
 * poststep.cu - per-step active-set update on uniform grids, the part of
 * PostStep at src/cipher.c:869-974.
 *
 *   k_post_prune : project phi of every cell with n > 1 onto the Gibbs
 *                  simplex (src/utility.c:578-603), write it back, and store
 *                  the pruned set {id : phi > TOL} in a scratch plane set;
 *                  cells with n == 1 get phi = 1.
 *   k_post_union : superset = own pruned set U pruned sets of the face
 *                  neighbours (sorted merge, src/utility.c:195-230); keep phi
 *                  and EX of surviving phases, zero phi and initialise EX of
 *                  new phases (SitepotentialExplicit of the material's c0 at
 *                  the cell temperature), write the superset.  A superset above P raises
 *                  the cap flag and leaves that cell's set unchanged.
 *
 * The projection and the TOL test run in FP64 for both precisions, so the
 * phase sets are decided by the same arithmetic as the reference.
 */
#include <cstdint>
#include <cuda_runtime.h>
#include "device_common.cuh"
#include "kernels.h"
#include "models.cuh"

namespace cipher {

template <int PM, typename R>
__device__ __forceinline__ void post_prune_cell(const PostArgs<R> &a, int64_t c)
{
    const int64_t S = a.stride;
    int n = a.as[c];
    if (n < 1 || n > a.P) {
        atomicOr(a.err, ERR_BADSET);
        a.pruned[c] = 0;
        return;
    }
    if (n == 1) {
        a.phi[c] = (R)1.0;
        a.pruned[c] = 1;
        a.pruned[S + c] = a.as[S + c];
        return;
    }
    double phi[PM], s[PM];
#pragma unroll
    for (int g = 0; g < PM; g++)
        if (g < n) { phi[g] = (double)a.phi[(int64_t)g * S + c]; s[g] = phi[g]; }
    /* sort a copy in descending order (insertion sort; n <= 16) */
    for (int i = 1; i < n; i++) {
        double v = s[i];
        int j = i - 1;
        while (j >= 0 && s[j] < v) { s[j + 1] = s[j]; j--; }
        s[j + 1] = v;
    }
    double sum = 0.0, tmax = 0.0;
    bool found = false;
    for (int i = 0; i < n - 1; i++) {
        sum += s[i];
        tmax = (sum - 1.0) / ((double)(i + 1));
        if (tmax >= s[i + 1]) { found = true; break; }
    }
    if (!found) tmax = (sum + s[n - 1] - 1.0) / ((double)n);
    int np = 0;
#pragma unroll
    for (int g = 0; g < PM; g++) {
        if (g < n) {
            double v = phi[g] - tmax > 0.0 ? phi[g] - tmax : 0.0;
            a.phi[(int64_t)g * S + c] = (R)v;
            if (v > CIPHER_TOL) {
                a.pruned[(int64_t)(1 + np) * S + c] = a.as[(int64_t)(1 + g) * S + c];
                np++;
            }
        }
    }
    a.pruned[c] = (uint16_t)np;
}

template <int PM, typename R>
__global__ void __launch_bounds__(256) k_post_prune(const PostArgs<R> a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    post_prune_cell<PM, R>(a, c);
}

/* out = a U b (sorted); returns the size, or P+1 if it would exceed P */
template <int PM>
__device__ __forceinline__ int merge_union(const uint16_t *sa, int na, const uint16_t *pl, int64_t S, int64_t nb,
                                           int nbn, uint16_t *out, int P)
{
    int i = 0, j = 0, n = 0;
    uint16_t b = nbn > 0 ? pl[S + nb] : 0;
    while (i < na || j < nbn) {
        uint16_t v;
        if (j >= nbn || (i < na && sa[i] < b)) {
            v = sa[i++];
        } else if (i >= na || b < sa[i]) {
            v = b;
            j++;
            if (j < nbn) b = pl[(int64_t)(1 + j) * S + nb];
        } else {
            v = sa[i++];
            j++;
            if (j < nbn) b = pl[(int64_t)(1 + j) * S + nb];
        }
        if (n >= P) return P + 1;
        out[n++] = v;
    }
    return n;
}

template <int DIM, int PM, typename R>
__device__ __forceinline__ void post_union_cell(const PostArgs<R> &a, int64_t c)
{
    const int64_t S = a.stride;
    int n = a.as[c];
    int ns = a.pruned[c];
    if (n < 1 || n > a.P || ns < 1 || ns > a.P) return;   /* flagged by k_post_prune */
    uint16_t sup[PM], tmp[PM];
    for (int k = 0; k < ns; k++) sup[k] = a.pruned[(int64_t)(1 + k) * S + c];

    /* union with the neighbours' pruned sets: over the faces of the cell
     * (src/cipher.c:930-945); the union does not depend on their order */
    auto unite = [&](int64_t nb) -> bool {
        if (nb == c) return true;
        int nbn = a.pruned[nb];
        if (nbn > a.P) nbn = a.P;
        int m = merge_union<PM>(sup, ns, a.pruned, S, nb, nbn, tmp, a.P);
        if (m > a.P) {
            atomicOr(a.err, ERR_CAP);
            return false;
        }
        for (int k = 0; k < m; k++) sup[k] = tmp[k];
        ns = m;
        return true;
    };
    if (a.fl.start) {
        for (int32_t e = a.fl.start[c]; e < a.fl.start[c + 1]; e++)
            if (!unite(a.fl.nbr[e] & 0x7fffffff)) return;
    } else {
        const int res[3] = {a.res[0], a.res[1], a.res[2]};
        const int64_t st[3] = {1, (int64_t)res[0], (int64_t)res[0] * res[1]};
        int co[3];
        co[0] = (int)(c % res[0]);
        co[1] = DIM > 1 ? (int)((c / res[0]) % res[1]) : 0;
        co[2] = DIM > 2 ? (int)(c / ((int64_t)res[0] * res[1])) : 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
#pragma unroll
            for (int side = 0; side < 2; side++) {
                int64_t nb;
                if (side == 0) {
                    if (co[d] > 0) nb = c - st[d];
                    else if (a.per[d] && res[d] > 1) nb = c + (int64_t)(res[d] - 1) * st[d];
                    else continue;
                } else {
                    if (co[d] < res[d] - 1) nb = c + st[d];
                    else if (a.per[d] && res[d] > 1) nb = c - (int64_t)(res[d] - 1) * st[d];
                    else continue;
                }
                if (!unite(nb)) return;
            }
        }
    }

    /* old (unpruned) set of this cell: phi survives for phases in the superset */
    uint16_t old[PM];
    for (int k = 0; k < n; k++) old[k] = a.as[(int64_t)(1 + k) * S + c];
    R phiss[PM];
    int from[PM];
    for (int g = 0; g < ns; g++) { phiss[g] = (R)0; from[g] = -1; }
    {
        int i = 0, j = 0;
        while (i < n && j < ns) {
            if (old[i] == sup[j]) { from[j] = i; i++; j++; }
            else if (old[i] < sup[j]) i++;
            else j++;
        }
    }
    for (int g = 0; g < ns; g++)
        if (from[g] >= 0) phiss[g] = a.phi[(int64_t)from[g] * S + c];
    /* explicit site potentials: survivors keep theirs, new phases start at
     * SitepotentialExplicit(c0) (src/cipher.c:953-964) */
    if (a.S > 0) {
        double exss[PM * 2 * CIPHER_MAXCP];
        const double T = (double)a.tm[c];
        for (int g = 0; g < ns; g++) {
            if (from[g] >= 0) {
                for (int q = 0; q < a.S; q++) exss[g * a.S + q] = a.ex[(int64_t)(from[g] * a.S + q) * S + c];
            } else if (a.chem.mat) {
                /* slots past the phase's own sites are never read; they start at 0 */
                const cipher_material &mat = material_of(a.chem, sup[g]);
                for (int q = 0; q < a.S; q++) exss[g * a.S + q] = 0.0;
                sitepot_explicit(a.chem, sup[g], mat.c0, T, &exss[g * a.S]);
            } else {
                for (int q = 0; q < a.S; q++) exss[g * a.S + q] = 0.0;
            }
        }
        for (int g = 0; g < ns; g++)
            for (int q = 0; q < a.S; q++) a.ex[(int64_t)(g * a.S + q) * S + c] = exss[g * a.S + q];
    }
    for (int g = 0; g < ns; g++) a.phi[(int64_t)g * S + c] = phiss[g];
    a.as[c] = (uint16_t)ns;
    for (int g = 0; g < ns; g++) a.as[(int64_t)(1 + g) * S + c] = sup[g];
}

template <int DIM, int PM, typename R>
__global__ void __launch_bounds__(256) k_post_union(const PostArgs<R> a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    post_union_cell<DIM, PM, R>(a, c);
}

/* face maps of cell c (cipher_b200.h, MAP): for each direction q = 2d+side
 * the neighbour's slot of every own phase, 15 where the neighbour lacks it
 * or where the face's L cell fails the phase-flux gate of src/cipher.c:277
 * (the L cell is the lower one of the face, as the reference enumerates
 * faces (c, c+e_d)).  Invalid sets raise ERR_BADSET. */
template <int DIM, typename R>
__device__ __forceinline__ void build_maps_cell(const PostArgs<R> &a, int64_t c)
{
    const int64_t S = a.stride;
    const int res[3] = {a.res[0], a.res[1], a.res[2]};
    const int64_t st[3] = {1, (int64_t)res[0], (int64_t)res[0] * res[1]};
    int co[3];
    co[0] = (int)(c % res[0]);
    co[1] = DIM > 1 ? (int)((c / res[0]) % res[1]) : 0;
    co[2] = DIM > 2 ? (int)(c / ((int64_t)res[0] * res[1])) : 0;
    const int n = a.as[c];
    bool ok = n >= 1 && n <= a.P;
    uint16_t own[CIPHER_PMAX];
    if (ok)
        for (int k = 0; k < n; k++) {
            own[k] = a.as[(int64_t)(1 + k) * S + c];
            if (a.npf > 0 && own[k] >= a.npf) ok = false;
        }
    if (!ok) atomicOr(a.err, ERR_BADSET);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
#pragma unroll
        for (int side = 0; side < 2; side++) {
            int64_t nb = -1;
            if (side == 0) {
                if (co[d] > 0) nb = c - st[d];
                else if (a.per[d] && res[d] > 1) nb = c + (int64_t)(res[d] - 1) * st[d];
            } else {
                if (co[d] < res[d] - 1) nb = c + st[d];
                else if (a.per[d] && res[d] > 1) nb = c - (int64_t)(res[d] - 1) * st[d];
            }
            uint64_t w = ~0ull;
            if (ok && nb >= 0) {
                const int nn = a.as[nb];
                if (nn >= 1 && nn <= a.P) {
                    const bool gate = side == 1 ? (n > 1 || own[0] > 1) : (nn > 1 || a.as[S + nb] > 1);
                    if (gate) {
                        int i = 0, j = 0;
                        while (i < n && j < nn) {
                            const uint16_t b = a.as[(int64_t)(1 + j) * S + nb];
                            if (own[i] == b) {
                                w &= ~(0xFull << (4 * i));
                                w |= (uint64_t)j << (4 * i);
                                i++;
                                j++;
                            } else if (own[i] < b) {
                                i++;
                            } else {
                                j++;
                            }
                        }
                    }
                }
            }
            a.maps[(int64_t)(2 * d + side) * S + c] = w;
        }
    }
}

template <int DIM, typename R>
__global__ void __launch_bounds__(256) k_build_maps(const PostArgs<R> a, int64_t c0, int64_t c1)
{
    const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    build_maps_cell<DIM, R>(a, c);
}

template <typename R>
static cudaError_t launch_maps(const PostArgs<R> &a, int dim, int64_t c0, int64_t c1, cudaStream_t s)
{
    if (!a.maps || c1 <= c0) return cudaSuccess;
    const int64_t blocks = (c1 - c0 + 255) / 256;
    if (dim == 1) k_build_maps<1, R><<<(unsigned)blocks, 256, 0, s>>>(a, c0, c1);
    else if (dim == 2) k_build_maps<2, R><<<(unsigned)blocks, 256, 0, s>>>(a, c0, c1);
    else k_build_maps<3, R><<<(unsigned)blocks, 256, 0, s>>>(a, c0, c1);
    return cudaGetLastError();
}

cudaError_t launch_build_maps(const PostArgs<double> &a, int dim, cudaStream_t s) { return launch_maps(a, dim, 0, a.ncells, s); }
cudaError_t launch_build_maps(const PostArgs<float> &a, int dim, cudaStream_t s) { return launch_maps(a, dim, 0, a.ncells, s); }
cudaError_t launch_build_maps_range(const PostArgs<double> &a, int dim, int64_t c0, int64_t c1, cudaStream_t s)
{
    return launch_maps(a, dim, c0, c1, s);
}
cudaError_t launch_build_maps_range(const PostArgs<float> &a, int dim, int64_t c0, int64_t c1, cudaStream_t s)
{
    return launch_maps(a, dim, c0, c1, s);
}

/* batched: block k of the list belongs to the domain whose range holds k */
template <typename R>
__device__ __forceinline__ int batch_post_domain(const BatchPost<R> &b, int64_t k)
{
    int lo = 0, hi = b.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&b.block_start[mid]) <= k) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int PM, typename R>
__global__ void __launch_bounds__(256) k_post_prune_batched(const BatchPost<R> b)
{
    const int inst = batch_post_domain(b, blockIdx.x);
    if (!b.active[inst]) return;
    const PostArgs<R> &a = b.args[inst];
    const int64_t c = (int64_t)(blockIdx.x - b.block_start[inst]) * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    post_prune_cell<PM, R>(a, c);
}

template <int DIM, int PM, typename R>
__global__ void __launch_bounds__(256) k_post_union_batched(const BatchPost<R> b)
{
    const int inst = batch_post_domain(b, blockIdx.x);
    if (!b.active[inst]) return;
    const PostArgs<R> &a = b.args[inst];
    const int64_t c = (int64_t)(blockIdx.x - b.block_start[inst]) * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    post_union_cell<DIM, PM, R>(a, c);
}

template <int DIM, typename R>
__global__ void __launch_bounds__(256) k_build_maps_batched(const BatchPost<R> b)
{
    const int inst = batch_post_domain(b, blockIdx.x);
    if (!b.active[inst]) return;
    const PostArgs<R> &a = b.args[inst];
    if (!a.maps) return;
    const int64_t c = (int64_t)(blockIdx.x - b.block_start[inst]) * blockDim.x + threadIdx.x;
    if (c >= a.ncells) return;
    build_maps_cell<DIM, R>(a, c);
}

template <typename R>
static cudaError_t launch_post_batched(const BatchPost<R> &b, int dim, cudaStream_t s)
{
    if (b.total < 1) return cudaSuccess;
    dim3 grid((unsigned)b.total), block(256);
    k_post_prune_batched<CIPHER_PMAX, R><<<grid, block, 0, s>>>(b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (dim == 1) k_post_union_batched<1, CIPHER_PMAX, R><<<grid, block, 0, s>>>(b);
    else if (dim == 2) k_post_union_batched<2, CIPHER_PMAX, R><<<grid, block, 0, s>>>(b);
    else k_post_union_batched<3, CIPHER_PMAX, R><<<grid, block, 0, s>>>(b);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (dim == 1) k_build_maps_batched<1, R><<<grid, block, 0, s>>>(b);
    else if (dim == 2) k_build_maps_batched<2, R><<<grid, block, 0, s>>>(b);
    else k_build_maps_batched<3, R><<<grid, block, 0, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_poststep_batched(const BatchPost<double> &b, int dim, cudaStream_t s) { return launch_post_batched(b, dim, s); }
cudaError_t launch_poststep_batched(const BatchPost<float> &b, int dim, cudaStream_t s) { return launch_post_batched(b, dim, s); }

template <typename R>
static cudaError_t launch_post(const PostArgs<R> &a, int dim, cudaStream_t s)
{
    int64_t blocks = (a.ncells + 255) / 256;
    dim3 grid((unsigned)blocks), block(256);
    k_post_prune<CIPHER_PMAX, R><<<grid, block, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (dim == 1) k_post_union<1, CIPHER_PMAX, R><<<grid, block, 0, s>>>(a);
    else if (dim == 2) k_post_union<2, CIPHER_PMAX, R><<<grid, block, 0, s>>>(a);
    else k_post_union<3, CIPHER_PMAX, R><<<grid, block, 0, s>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return launch_maps(a, dim, 0, a.ncells, s);
}

cudaError_t launch_poststep(const PostArgs<double> &a, int dim, cudaStream_t s) { return launch_post(a, dim, s); }
cudaError_t launch_poststep(const PostArgs<float> &a, int dim, cudaStream_t s) { return launch_post(a, dim, s); }

}  // namespace cipher
