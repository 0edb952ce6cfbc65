// memory.cu -- device memory of the library: one stream-ordered pool per device that keeps freed
// memory reserved for the library's next allocations.
//
// A solve handle owns several GB (matrices, factor, layouts, sort buffers of the analysis), and
// the one-shot entry point and GUI-style callers create and destroy one per solve. With plain
// cudaMalloc / cudaFree every such cycle maps and unmaps that memory again: on a B200 the first
// allocation of a handle's buffers took about 0.2 s and a handle's frees up to 0.5 s. The pool
// (cudaMemPoolCreate, release threshold at its maximum) hands the same memory back instead;
// maille_gpu_trim_memory returns what is unused to the device.
//
// Ordering: an allocation is made on the library's allocation stream and waited for before it is
// returned, so it is ready for any stream; a free first waits for the device to be idle (the same
// implicit synchronisation cudaFree performs), so no kernel still uses the memory when the pool
// may hand it out again.

#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "cuda_host.hpp"

namespace maille {
namespace {

struct DevicePool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
};

std::mutex g_pool_mutex;
std::vector<DevicePool> g_pools;

DevicePool& pool_of_current_device() {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if ((int)g_pools.size() <= dev) g_pools.resize(dev + 1);
    DevicePool& d = g_pools[dev];
    if (!d.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        CK(cudaMemPoolCreate(&d.pool, &props));
        uint64_t keep = UINT64_MAX;
        CK(cudaMemPoolSetAttribute(d.pool, cudaMemPoolAttrReleaseThreshold, &keep));
        CK(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
    }
    return d;
}

}  // namespace

void* device_alloc(size_t bytes) {
    DevicePool& d = pool_of_current_device();
    void* p = nullptr;
    CK(cudaMallocFromPoolAsync(&p, bytes, d.pool, d.stream));
    CK(cudaStreamSynchronize(d.stream));
    return p;
}

void device_free(void* p) {
    if (!p) return;
    DevicePool& d = pool_of_current_device();
    cudaDeviceSynchronize();
    cudaFreeAsync(p, d.stream);
    cudaStreamSynchronize(d.stream);
}

void device_free_all(const std::vector<void*>& ps) {
    bool any = false;
    for (void* p : ps) any = any || p != nullptr;
    if (!any) return;
    DevicePool& d = pool_of_current_device();
    for (void* p : ps)
        if (p) cudaFreeAsync(p, d.stream);
    cudaStreamSynchronize(d.stream);
}

namespace {

// Small pinned host slots (a handle's scalar read-back, a cancel flag). Each cudaFreeHost waits for
// every device, and a handle's destruction took tens of milliseconds in two of them; the slots are
// carved from mapped, portable chunks that stay allocated for the process, so a slot's device
// address is its host address on every device (unified addressing).
constexpr size_t kPinnedSlot = 256;
constexpr size_t kPinnedChunk = 64 * 1024;
std::mutex g_pinned_mutex;
std::vector<void*> g_pinned_free;

}  // namespace

void* pinned_slot_alloc(size_t bytes) {
    if (bytes > kPinnedSlot) throw CudaFailure{"pinned_slot_alloc: more than 256 bytes asked"};
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    if (g_pinned_free.empty()) {
        void* chunk = nullptr;
        CK(cudaHostAlloc(&chunk, kPinnedChunk, cudaHostAllocMapped | cudaHostAllocPortable));
        for (size_t off = kPinnedChunk; off >= kPinnedSlot; off -= kPinnedSlot)
            g_pinned_free.push_back(static_cast<char*>(chunk) + off - kPinnedSlot);
    }
    void* p = g_pinned_free.back();
    g_pinned_free.pop_back();
    std::memset(p, 0, kPinnedSlot);
    return p;
}

void pinned_slot_free(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    g_pinned_free.push_back(p);
}

int device_sms() {
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cached[kMaxDevices];
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        return sms;
    }
    int sms = cached[dev].load(std::memory_order_relaxed);
    if (sms <= 0) {
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        cached[dev].store(sms, std::memory_order_relaxed);
    }
    return sms;
}

int32_t trim_device_memory(int device) {
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return -1;
    int32_t status = 0;
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        if (device < (int)g_pools.size() && g_pools[device].pool) {
            cudaDeviceSynchronize();
            status = cudaMemPoolTrimTo(g_pools[device].pool, 0) == cudaSuccess ? 0 : -1;
        }
    }
    cudaSetDevice(prev);
    return status;
}

}  // namespace maille
