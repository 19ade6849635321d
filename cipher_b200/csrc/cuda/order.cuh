/*
 * order.cuh - cells grouped by class for kernels whose per-cell work
 * depends on the class (the set size, the material of a single phase):
 * lanes of a warp then run the same loops.
 *
 * Counting sort within segments of kOrderSegBlocks blocks of 256 cells
 * (16 384 cells): a segment's cells stay in the segment's own range of the
 * order, class by class, and within a class in grid order.  Walking the
 * order therefore sweeps the domain once, segment after segment, so the
 * neighbour data a segment's gathers touch is still in L2 (grouping over
 * the whole domain instead sweeps it once per class, and L2 cannot hold the
 * state between sweeps).
 *   k_order_count : per block, the count of each class (counts[k][block]);
 *   k_order_scan  : one block per segment: each class's start in the
 *                   segment plus the exclusive prefix over the segment's
 *                   blocks (counts become offsets);
 *   k_order_place : per block, each cell at its class's block offset plus
 *                   its rank among the block's cells of that class (ballots).
 * Key is a functor int(int64_t cell) returning a class in [0, nclass).
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "kernels.h"

namespace cipher {

constexpr int kOrderBlock = 256;
constexpr int kOrderSegBlocks = 64;

struct OrderBuf {
    int32_t *order;        /* [ncells] */
    int32_t *counts;       /* [kOrderClasses][nblocks]: counts, then offsets */
    int32_t *totals;       /* unused by the segmented sort (kept for the buffer layout) */
    int nclass;
    int64_t ncells;
};

template <typename Key>
__global__ void __launch_bounds__(kOrderBlock) k_order_count(const OrderBuf o, const Key key)
{
    __shared__ int cnt[kOrderClasses];
    if (threadIdx.x < kOrderClasses) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < o.ncells) atomicAdd(&cnt[key(c)], 1);
    __syncthreads();
    if (threadIdx.x < o.nclass) o.counts[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

/* grid = segments; nblocks = the count kernel's grid */
static __global__ void __launch_bounds__(kOrderClasses) k_order_scan(const OrderBuf o, int nblocks)
{
    __shared__ int tot[kOrderClasses];
    const int k = threadIdx.x;
    const int b0 = blockIdx.x * kOrderSegBlocks;
    const int b1 = b0 + kOrderSegBlocks < nblocks ? b0 + kOrderSegBlocks : nblocks;
    int t = 0;
    if (k < o.nclass)
        for (int b = b0; b < b1; b++) t += o.counts[(int64_t)k * nblocks + b];
    tot[k] = t;
    __syncthreads();
    if (k < o.nclass) {
        int start = b0 * kOrderBlock;                /* cells of the earlier segments */
        for (int j = 0; j < k; j++) start += tot[j];
        for (int b = b0; b < b1; b++) {
            int32_t *p = &o.counts[(int64_t)k * nblocks + b];
            const int v = *p;
            *p = start;
            start += v;
        }
    }
}

template <typename Key>
__global__ void __launch_bounds__(kOrderBlock) k_order_place(const OrderBuf o, const Key key)
{
    __shared__ int wcnt[kOrderBlock / 32][kOrderClasses];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int cls = c < o.ncells ? key(c) : -1;
    int rank = 0;
    for (int k = 0; k < o.nclass; k++) {
        const unsigned m = __ballot_sync(0xffffffffu, cls == k);
        if (cls == k) rank = __popc(m & ((1u << lane) - 1u));
        if (lane == 0) wcnt[warp][k] = __popc(m);
    }
    __syncthreads();
    if (cls >= 0) {
        int off = o.counts[(int64_t)cls * gridDim.x + blockIdx.x];
        for (int w = 0; w < warp; w++) off += wcnt[w][cls];
        o.order[off + rank] = (int32_t)c;
    }
}

/* the three passes on stream s */
template <typename Key>
inline void launch_order(const OrderBuf &o, const Key &key, cudaStream_t s)
{
    const unsigned nb = (unsigned)((o.ncells + kOrderBlock - 1) / kOrderBlock);
    const unsigned nseg = (nb + kOrderSegBlocks - 1) / kOrderSegBlocks;
    k_order_count<Key><<<nb, kOrderBlock, 0, s>>>(o, key);
    k_order_scan<<<nseg, kOrderClasses, 0, s>>>(o, (int)nb);
    k_order_place<Key><<<nb, kOrderBlock, 0, s>>>(o, key);
}

}  // namespace cipher
