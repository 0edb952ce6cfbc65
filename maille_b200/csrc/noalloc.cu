// noalloc.cu -- y = A x and x . y for a 3x3-block CSR matrix, without allocating device memory.
//
// For callers that cannot allocate device memory at the point where they need this product: code
// running while a stream is being captured into a CUDA graph (cudaMalloc is not allowed there),
// code in a plugin whose host framework owns every device allocation, or a real-time loop that
// must not allocate. Such callers hold the matrix and the vectors in device memory they already
// own; the only extra memory the product needs, the per-block partial sums and the finishing
// ticket of the deterministic dot-product reduction, lives in a file-scope device array that the
// library carries.
//
// The array is shared by every call in the process: calls that run at the same time on the GPU
// (from two threads, or on two streams without ordering) race on it and must not overlap. The
// array keeps the last call's contents, so each call clears the ticket before its kernel runs.
//
// Set-up: the first call on a device looks up the array's device address with that device current
// (cudaGetSymbolAddress) and caches it. Make that first call before starting any stream capture.

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/maille_gpu.h"
#include "reduce.cuh"

namespace maille {
extern std::atomic<long long> g_kernel_launches;
void set_last_error(const std::string& message);
}

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaWarps = kNaThreads / 32;
constexpr int kNaMaxBlocks = 1024;  // partial sums held in the scratch array

// Scratch of the reduction: kNaMaxBlocks partial sums, then the ticket counter: 8200 bytes (8192
// + 4, padded to the struct's 8-byte alignment), placed at a 256-byte boundary.
struct NoallocScratch {
    double partials[kNaMaxBlocks];
    unsigned int ticket;
};
static_assert(sizeof(NoallocScratch) == 8200, "the scratch size stated in maille_gpu.h");
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

// [a, a + na) and [b, b + nb) share a byte
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
    const uintptr_t pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    return pa < pb + nb && pb < pa + na;
}

// y_I = sum_J A_IJ x_J for block rows I (one warp per row, lanes over the row's blocks), the
// partial sums of x . y per block in the scratch, the ordered total by the last block to finish.
__global__ void __launch_bounds__(kNaThreads) k_bsr3_spmv_dot(int64_t nb, const int64_t* __restrict__ row_ptr,
                                                              const int32_t* __restrict__ col,
                                                              const double* __restrict__ vals,
                                                              const double* __restrict__ x,
                                                              double* __restrict__ y, double* xy,
                                                              NoallocScratch* scratch) {
    __shared__ double sh[kNaWarps];
    const int lane = threadIdx.x & 31;
    double loc = 0.0;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nb;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int64_t p = row_ptr[i] + lane; p < row_ptr[i + 1]; p += 32) {
            const double* v = vals + 9 * p;
            const int64_t j = col[p];
            const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
            a0 += v[0] * x0 + v[1] * x1 + v[2] * x2;
            a1 += v[3] * x0 + v[4] * x1 + v[5] * x2;
            a2 += v[6] * x0 + v[7] * x1 + v[8] * x2;
        }
        a0 = maille::warp_sum(a0);
        a1 = maille::warp_sum(a1);
        a2 = maille::warp_sum(a2);
        if (lane == 0) {
            y[3 * i] = a0;
            y[3 * i + 1] = a1;
            y[3 * i + 2] = a2;
            loc += x[3 * i] * a0 + x[3 * i + 1] * a1 + x[3 * i + 2] * a2;
        }
    }
    if (maille::publish_partial(loc, scratch->partials, &scratch->ticket, sh)) {
        const double tot = maille::gather_sum(scratch->partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            *xy = tot;
            scratch->ticket = 0;
        }
    }
}

std::mutex g_na_mutex;
NoallocScratch* g_na_ptr[64] = {nullptr};

}  // namespace

extern "C" int32_t maille_gpu_bsr3_spmv_dot_noalloc(int32_t device, int64_t n_block_rows,
                                                    const int64_t* row_ptr, const int32_t* col,
                                                    const double* vals, const double* x, double* y,
                                                    double* xy, void* stream) {
    maille::set_last_error("");
    if (n_block_rows < 0 || n_block_rows > MAILLE_NOALLOC_MAX_BLOCK_ROWS) {
        maille::set_last_error("n_block_rows " + std::to_string(n_block_rows) +
                               " is outside [0, MAILLE_NOALLOC_MAX_BLOCK_ROWS = " +
                               std::to_string((long long)MAILLE_NOALLOC_MAX_BLOCK_ROWS) + "]");
        return MAILLE_INVALID_INPUT;
    }
    if (!row_ptr || !col || !vals || !x || !y || !xy) {
        maille::set_last_error("null device pointer");
        return MAILLE_INVALID_INPUT;
    }
    // warps write rows of y while others still read x: an in-place or overlapping call would
    // read half-updated entries (the kernel's pointers are __restrict__)
    const size_t vec_bytes = 3 * (size_t)n_block_rows * sizeof(double);
    if (overlaps(x, vec_bytes, y, vec_bytes) || overlaps(xy, sizeof(double), y, vec_bytes) ||
        overlaps(xy, sizeof(double), x, vec_bytes)) {
        maille::set_last_error("x, y and xy must not overlap");
        return MAILLE_INVALID_INPUT;
    }
    if (device < 0 || device >= 64) {
        maille::set_last_error("device ordinal out of range");
        return MAILLE_INVALID_INPUT;
    }
    int previous = 0;
    if (cudaGetDevice(&previous) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        maille::set_last_error("cannot select CUDA device " + std::to_string(device));
        return MAILLE_CUDA_ERROR;
    }
    NoallocScratch* scratch = nullptr;
    {
        // one-time set-up on this device: the device address of the scratch array
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!g_na_ptr[device]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                maille::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                cudaSetDevice(previous);
                return MAILLE_CUDA_ERROR;
            }
            g_na_ptr[device] = static_cast<NoallocScratch*>(p);
        }
        scratch = g_na_ptr[device];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int32_t status = MAILLE_OK;
    if (cudaMemsetAsync(&scratch->ticket, 0, sizeof(unsigned int), st) != cudaSuccess) {
        maille::set_last_error("cannot clear the reduction ticket on the given stream");
        status = MAILLE_CUDA_ERROR;
    } else if (n_block_rows == 0) {
        if (cudaMemsetAsync(xy, 0, sizeof(double), st) != cudaSuccess) {
            maille::set_last_error("cannot clear xy on the given stream");
            status = MAILLE_CUDA_ERROR;
        }
    } else {
        int64_t blocks = (n_block_rows + kNaWarps - 1) / kNaWarps;
        if (blocks > kNaMaxBlocks) blocks = kNaMaxBlocks;
        k_bsr3_spmv_dot<<<(unsigned)blocks, kNaThreads, 0, st>>>(n_block_rows, row_ptr, col, vals, x,
                                                                 y, xy, scratch);
        maille::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            maille::set_last_error(std::string("kernel launch: ") + cudaGetErrorString(e));
            status = MAILLE_CUDA_ERROR;
        }
    }
    cudaSetDevice(previous);
    return status;
}
