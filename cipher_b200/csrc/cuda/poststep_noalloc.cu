/*
 * poststep_noalloc.cu - the per-step active-set update for callers that
 * cannot allocate device memory.
 *
 * Some hosts cannot call cudaMalloc: a solver embedded in another
 * application that owns the device heap, a fixed-footprint service that
 * reserves all its memory up front, or code running where allocation is
 * forbidden after start-up.  For them cipher_poststep_noalloc runs the same
 * two kernels as cipher_poststep (projection/pruning, then the neighbour
 * union), but its scratch - the pruned active sets of every cell - lives in a
 * file-scope device array of fixed size instead of a context allocation, and
 * it needs no context at all: the caller describes the grid and the state
 * layout and passes the state vector.
 *
 * Limits and behaviour:
 *   - scratch holds (P+1) * stride uint16 values, at most
 *     CIPHER_NOALLOC_MAX_PRUNED (4 Mi values, 8 MiB); larger grids are
 *     rejected with CIPHER_E_ARG.  Every GPU that loads the library holds
 *     the 8 MiB until the process exits.
 *   - the first call on a device looks up the array's device address with
 *     that device current; make that first call before any stream capture.
 *   - all calls share the one array and its error word: calls that overlap
 *     on the GPU (other streams, other host threads) race.  The error word is
 *     cleared at the start of each call; the pruned sets are fully rewritten.
 *   - no cudaMalloc, cudaFree or allocating library call is made.
 *   - with chemistry (S > 0) the caller passes device copies of the
 *     problem's material table and phase-material mapping, so that a phase
 *     that joins a cell starts at SitepotentialExplicit(c0, T of the cell),
 *     the same branch cipher_poststep takes (src/cipher.c:953-964).
 */
#include <cstdint>
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "device_common.cuh"
#include "kernels.h"

#define CIPHER_NOALLOC_MAX_PRUNED (4u << 20)
#define CIPHER_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) uint16_t g_noalloc_pruned[CIPHER_NOALLOC_MAX_PRUNED];
static __device__ __align__(256) int g_noalloc_flags;

namespace {

struct NoallocSymbols {
    uint16_t *pruned = nullptr;
    int *flags = nullptr;
    bool ready = false;
};

std::mutex g_noalloc_mutex;
NoallocSymbols g_noalloc_syms[CIPHER_NOALLOC_MAX_DEVICES];

/* device addresses of the static scratch for the current device */
cudaError_t noalloc_symbols(int device, NoallocSymbols &out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocSymbols &s = g_noalloc_syms[device];
    if (!s.ready) {
        cudaError_t e = cudaGetSymbolAddress((void **)&s.pruned, g_noalloc_pruned);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress((void **)&s.flags, g_noalloc_flags);
        if (e != cudaSuccess) return e;
        s.ready = true;
    }
    out = s;
    return cudaSuccess;
}

template <typename R>
cipher::PostArgs<R> noalloc_args(const cipher_grid_desc *g, void *X, const NoallocSymbols &sy)
{
    cipher::PostArgs<R> a;
    memset(&a, 0, sizeof(a));
    char *x = (char *)X;
    a.ncells = g->layout.ncells;
    a.stride = g->layout.stride;
    for (int d = 0; d < 3; d++) {
        a.res[d] = d < g->dim ? g->res[d] : 1;
        a.per[d] = d < g->dim ? (g->periodic[d] && g->res[d] > 1) : 0;
    }
    a.P = g->layout.pf_size;
    a.S = g->ex_per_phase;
    a.npf = g->npf;
    a.as = (uint16_t *)(x + g->layout.as_offset);
    /* the face maps of the layout, when it has them, are rebuilt as well */
    a.maps = g->layout.map_planes == g->layout.pf_size ? (uint32_t *)(x + g->layout.map_offset) : nullptr;
    a.phi = (R *)(x + g->layout.pf_offset);
    a.ex = (double *)(x + g->layout.ex_offset);
    a.tm = (const R *)(x + g->layout.tm_offset);
    a.pruned = sy.pruned;
    if (g->ex_per_phase > 0) {
        a.chem.mat = g->materials;
        a.chem.pmm = g->phasematerialmapping;
        a.chem.ncp = g->ncp;
        a.chem.ndp = g->ncp - 1;
        a.chem.nmat = g->nmat;
    }
    a.err = sy.flags;
    return a;
}

}  // namespace

extern "C" int cipher_poststep_noalloc(const cipher_grid_desc *g, void *X, void *stream)
{
    if (!g || !X) return CIPHER_E_ARG;
    if (g->dim < 1 || g->dim > 3) return CIPHER_E_ARG;
    const int P = g->layout.pf_size;
    if (P < 1 || P > CIPHER_MAXAP || g->layout.stride < g->layout.ncells || g->layout.ncells < 1) return CIPHER_E_ARG;
    int64_t cells = 1;
    for (int d = 0; d < g->dim; d++) {
        if (g->res[d] < 1) return CIPHER_E_ARG;
        cells *= g->res[d];
    }
    if (cells != g->layout.ncells) return CIPHER_E_ARG;
    if (g->npf < 1 || g->npf > 65535) return CIPHER_E_ARG;
    /* the face maps (one word plane per slot) are rebuilt when the layout has
     * them; any other plane count is a foreign layout */
    if (g->layout.map_planes != 0 && g->layout.map_planes != P) return CIPHER_E_ARG;
    /* explicit site potentials: S per phase, at most two sublattices of ncp-1 potentials */
    const int S = g->ex_per_phase;
    if (S < 0 || S > 2 * CIPHER_MAXCP) return CIPHER_E_ARG;
    if (g->layout.ex_size != P * S) return CIPHER_E_ARG;
    if (S > 0) {
        if (!g->materials || !g->phasematerialmapping) return CIPHER_E_ARG;
        if (g->ncp < 2 || g->ncp > CIPHER_MAXCP || g->nmat < 1 || S > 2 * (g->ncp - 1)) return CIPHER_E_ARG;
    }
    if (g->layout.precision != CIPHER_PREC_FP64 && g->layout.precision != CIPHER_PREC_MIXED) return CIPHER_E_ARG;
    /* the static scratch holds (P+1) planes of `stride` pruned-set entries */
    if ((uint64_t)(P + 1) * (uint64_t)g->layout.stride > CIPHER_NOALLOC_MAX_PRUNED) return CIPHER_E_ARG;

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= CIPHER_NOALLOC_MAX_DEVICES)
        return CIPHER_E_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        /* the scratch looked up below is the current device's */
        int sdev = -1;
        if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) return CIPHER_E_CUDA;
        if (sdev != device) return CIPHER_E_ARG;
    }
    NoallocSymbols sy;
    if (noalloc_symbols(device, sy) != cudaSuccess) return CIPHER_E_CUDA;
    if (cudaMemsetAsync(sy.flags, 0, sizeof(int), s) != cudaSuccess) return CIPHER_E_CUDA;
    cudaError_t e;
    if (g->layout.precision == CIPHER_PREC_FP64)
        e = cipher::launch_poststep(noalloc_args<double>(g, X, sy), g->dim, s);
    else
        e = cipher::launch_poststep(noalloc_args<float>(g, X, sy), g->dim, s);
    if (e != cudaSuccess) return CIPHER_E_CUDA;
    int flags = 0;
    if (cudaMemcpyAsync(&flags, sy.flags, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CIPHER_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CIPHER_E_CUDA;
    if (flags & cipher::ERR_CAP) return CIPHER_E_CAP;
    if (flags & cipher::ERR_BADSET) return CIPHER_E_ARG;
    return CIPHER_OK;
}
