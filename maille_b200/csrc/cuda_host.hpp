// cuda_host.hpp -- host-side CUDA helpers shared by the handle and batch drivers: error
// checking that throws to the C ABI boundary, device allocation and upload, a wall clock.
#pragma once

#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

namespace maille {

// A named range on a profiler's host timeline (NVTX, header-only: without a tool attached the
// calls do nothing). One per entry point and per major phase.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

struct CudaFailure {
    std::string what;
};

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            throw ::maille::CudaFailure{std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

inline double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Device memory from the library's per-device pool (memory.cu): an allocation is ready for any
// stream when it returns; a free waits for the device to be idle, like cudaFree.
void* device_alloc(size_t bytes);
void device_free(void* p);
// Frees every non-null pointer of `ps` on the pool's stream and waits for it; the caller has
// synchronised every stream that used them (a handle's destructor: its own stream).
void device_free_all(const std::vector<void*>& ps);
// Returns the pool's unused memory of `device` to the device (0, or -1 on a CUDA error).
int32_t trim_device_memory(int device);
// A zeroed pinned host slot of at most 256 bytes, mapped and portable (its device address equals
// its host address); slots are reused, never returned to the driver.
void* pinned_slot_alloc(size_t bytes);
void pinned_slot_free(void* p);
// Streaming multiprocessors of the current device (cudaDevAttrMultiProcessorCount, cached per
// device): grid caps are multiples of it.
int device_sms();

template <typename T>
T* dalloc(size_t n) {
    if (n == 0) n = 1;
    return static_cast<T*>(device_alloc(n * sizeof(T)));
}

template <typename T>
T* dupload(const T* src, size_t n, cudaStream_t st) {
    T* d = dalloc<T>(n);
    if (n && src) CK(cudaMemcpyAsync(d, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return d;
}

inline void dfree(void* p) { device_free(p); }

constexpr double kDefaultTol = 1e-12;      // iterative.rs:9
constexpr int32_t kDefaultMaxIter = 10000;  // iterative.rs:11
constexpr double kShifts[6] = {0.0, 1e-3, 1e-2, 1e-1, 1.0, 10.0};  // iterative.rs:14

void set_last_error(const std::string& message);

}  // namespace maille
