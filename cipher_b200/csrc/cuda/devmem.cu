/*
 * devmem.cu - device memory of contexts, steppers, batches and served
 * requests.
 *
 * Long-lived buffers come from one stream-ordered memory pool per device
 * that keeps freed blocks for reuse (release threshold: unlimited), so that
 * a server admitting and retiring requests many times a second reuses
 * memory instead of paying cudaMalloc/cudaFree each time: cudaFree waits for
 * the whole device, a pool free does not.
 *
 * dev_alloc returns memory that any stream may use at once (the pool's own
 * stream is synchronised after the allocation).  dev_free returns a block to
 * the pool without waiting: the caller guarantees that no queued or running
 * work still uses it (the destroy paths synchronise the device first, as
 * cudaFree would have).  cipher_pool_trim hands pooled blocks back to the
 * driver.
 */
#include <cstdint>
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>
#include "cipher_b200.h"
#include "kernels.h"

namespace cipher {

namespace {

constexpr int kMaxDevices = 64;

struct DevicePool {
    bool ready = false;
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
};

std::mutex g_pool_mutex;
DevicePool g_pools[kMaxDevices];

cudaError_t pool_of(int device, DevicePool *&out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    DevicePool &p = g_pools[device];
    if (!p.ready) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaError_t e = cudaMemPoolCreate(&p.pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
        int cur = 0;
        if ((e = cudaGetDevice(&cur)) != cudaSuccess) return e;
        if (cur != device && (e = cudaSetDevice(device)) != cudaSuccess) return e;
        e = cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking);
        if (cur != device) cudaSetDevice(cur);
        if (e != cudaSuccess) return e;
        p.ready = true;
    }
    out = &p;
    return cudaSuccess;
}

}  // namespace

cudaError_t dev_alloc(void **ptr, size_t bytes)
{
    *ptr = nullptr;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    DevicePool *p = nullptr;
    if ((e = pool_of(device, p)) != cudaSuccess) return e;
    if ((e = cudaMallocFromPoolAsync(ptr, bytes, p->pool, p->stream)) != cudaSuccess) {
        *ptr = nullptr;
        return e;
    }
    e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(*ptr, p->stream);
        *ptr = nullptr;
    }
    return e;
}

void dev_free(void *ptr)
{
    if (!ptr) return;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return;
    }
    DevicePool *p = nullptr;
    if (pool_of(at.device, p) != cudaSuccess) return;
    cudaFreeAsync(ptr, p->stream);
}

/* pinned host words (a context's error flag, a stepper's norm): slabs of
 * pinned memory carved into 64-byte slots, so that creating and destroying
 * contexts does not pay cudaMallocHost/cudaFreeHost each time */
namespace {
constexpr int kSlotBytes = 64, kSlabSlots = 1024;
std::mutex g_pinned_mutex;
struct PinnedSlot { PinnedSlot *next; };
PinnedSlot *g_pinned_free = nullptr;
}  // namespace

cudaError_t pinned_word_alloc(void **ptr)
{
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    if (!g_pinned_free) {
        char *slab = nullptr;
        cudaError_t e = cudaMallocHost((void **)&slab, (size_t)kSlotBytes * kSlabSlots);
        if (e != cudaSuccess) { *ptr = nullptr; return e; }
        for (int i = kSlabSlots - 1; i >= 0; i--) {
            PinnedSlot *s = (PinnedSlot *)(slab + (size_t)i * kSlotBytes);
            s->next = g_pinned_free;
            g_pinned_free = s;
        }
    }
    PinnedSlot *s = g_pinned_free;
    g_pinned_free = s->next;
    memset((void *)s, 0, kSlotBytes);
    *ptr = s;
    return cudaSuccess;
}

void pinned_word_free(void *ptr)
{
    if (!ptr) return;
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    PinnedSlot *s = (PinnedSlot *)ptr;
    s->next = g_pinned_free;
    g_pinned_free = s;
}

}  // namespace cipher

extern "C" int cipher_pool_trim(int device)
{
    cipher::DevicePool *p = nullptr;
    if (cipher::pool_of(device, p) != cudaSuccess) return CIPHER_E_CUDA;
    if (cudaStreamSynchronize(p->stream) != cudaSuccess) return CIPHER_E_CUDA;
    if (cudaMemPoolTrimTo(p->pool, 0) != cudaSuccess) return CIPHER_E_CUDA;
    return CIPHER_OK;
}
