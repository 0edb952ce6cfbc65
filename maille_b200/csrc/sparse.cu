// sparse.cu -- SELL 3x3-block SpMV (standalone), PCG set-up kernels and the layout fills.
// Layout and conventions: sparse.cuh. Reductions: reduce.cuh (deterministic).

#include <atomic>
#include <cmath>

#include "cuda_host.hpp"
#include "reduce.cuh"
#include "sparse.cuh"

namespace maille {

extern std::atomic<long long> g_kernel_launches;

namespace {

constexpr int kThr = 256;
constexpr int kWarp = kThr / 32;
// blocks per SM at most for the grid-stride kernels (the grid is this times the SM count)
constexpr int kMaxBlocksPerSm = 8;

inline int grid_for(int64_t items, int per_block, int blocks_per_sm = kMaxBlocksPerSm) {
    int64_t g = (items + per_block - 1) / per_block;
    const int64_t cap = (int64_t)blocks_per_sm * device_sms();
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

inline void counted() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }

// 4 consecutive values from a 16-byte aligned address
__device__ __forceinline__ void load4(const float* p, float v[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void load4(const double* p, double v[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p + 2));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// the 3 components of node c of a padded vector
__device__ __forceinline__ void node3(const float* x, int32_t c, float& a, float& b, float& d) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(x + 4 * (int64_t)c));
    a = q.x; b = q.y; d = q.z;
}
__device__ __forceinline__ void node3(const double* x, int32_t c, double& a, double& b, double& d) {
    const double2 q = __ldg(reinterpret_cast<const double2*>(x + 4 * (int64_t)c));
    a = q.x; b = q.y; d = __ldg(x + 4 * (int64_t)c + 2);
}
// plain (coherent) read of node c, for vectors written earlier in the same launch sequence
template <typename T>
__device__ __forceinline__ void node3_rw(const T* x, int64_t i, T& a, T& b, T& d) {
    a = x[4 * i]; b = x[4 * i + 1]; d = x[4 * i + 2];
}
// the 4 padded entries of node i (plain loads / stores, 128-bit for FP32, 2 x 128-bit for FP64)
struct F4 {
    double v[4];
};
__device__ __forceinline__ F4 ld4(const float* x, int64_t i) {
    const float4 q = *reinterpret_cast<const float4*>(x + 4 * i);
    return F4{{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ F4 ld4(const double* x, int64_t i) {
    const double2 a = *reinterpret_cast<const double2*>(x + 4 * i);
    const double2 b = *reinterpret_cast<const double2*>(x + 4 * i + 2);
    return F4{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* x, int64_t i, const F4& f) {
    *reinterpret_cast<float4*>(x + 4 * i) = make_float4((float)f.v[0], (float)f.v[1], (float)f.v[2], (float)f.v[3]);
}
__device__ __forceinline__ void st4(double* x, int64_t i, const F4& f) {
    *reinterpret_cast<double2*>(x + 4 * i) = make_double2(f.v[0], f.v[1]);
    *reinterpret_cast<double2*>(x + 4 * i + 2) = make_double2(f.v[2], f.v[3]);
}
template <typename T>
__device__ __forceinline__ void store_node(T* x, int64_t i, T a, T b, T d) {
    x[4 * i] = a; x[4 * i + 1] = b; x[4 * i + 2] = d; x[4 * i + 3] = T(0);
}

// acc += this lane's 4 slots of step g with columns c4: V_b x[col_b] (3x3 blocks)
template <typename T>
__device__ __forceinline__ void step_accum(const T* __restrict__ vals, int4 c4, int64_t g,
                                           const T* __restrict__ x, int lane, int32_t pad, T& a0, T& a1,
                                           T& a2) {
    const T* V = vals + g * 9 * kStepSlots + 4 * lane;
    T v[9][4];
#pragma unroll
    for (int k = 0; k < 9; ++k) load4(V + k * kStepSlots, v[k]);
    const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        T x0 = 0, x1 = 0, x2 = 0;
        if (cc[j] != pad) node3(x, cc[j], x0, x1, x2);  // padding slots: zero values, no load
        a0 += v[0][j] * x0 + v[1][j] * x1 + v[2][j] * x2;
        a1 += v[3][j] * x0 + v[4][j] * x1 + v[5][j] * x2;
        a2 += v[6][j] * x0 + v[7][j] * x1 + v[8][j] * x2;
    }
}

// acc += sum over the slice steps [g0, g1) of this lane's slots
template <typename T>
__device__ __forceinline__ void slice_accum(const T* __restrict__ vals,
                                            const int32_t* __restrict__ col, int64_t g0, int64_t g1,
                                            const T* __restrict__ x, int lane, int32_t pad, T& a0,
                                            T& a1, T& a2) {
    // each step's columns are fetched one step ahead, so its gathers wait on L2 only
    int4 cnext = __ldg(reinterpret_cast<const int4*>(col + g0 * kStepSlots + 4 * lane));
    for (int64_t g = g0; g < g1; ++g) {
        const int4 c4 = cnext;
        if (g + 1 < g1) cnext = __ldg(reinterpret_cast<const int4*>(col + (g + 1) * kStepSlots + 4 * lane));
        step_accum<T>(vals, c4, g, x, lane, pad, a0, a1, a2);
    }
}

template <typename T, int LPR>
__device__ __forceinline__ void row_reduce(T& a0, T& a1, T& a2) {
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
}

// ap = K p (Csr::multiply, iterative.rs:131-142, as a gather on the full symmetric pattern) on its
// own: the handle's multiply entry point and the SpMV timing launches. (Inside the solve the SpMV
// is a phase of the persistent kernel, persist.cu.)
template <typename T, int LPR>
__global__ void __launch_bounds__(kThr) k_spmv(SellDev A, const T* __restrict__ vals,
                                                const T* __restrict__ p, T* __restrict__ ap) {
    const int lane = threadIdx.x & 31, r = lane / LPR, q = lane % LPR;
    constexpr int S = 32 / LPR;
    for (int32_t sl = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); sl < A.nslices;
         sl += (int32_t)((gridDim.x * blockDim.x) >> 5)) {
        T a0 = 0, a1 = 0, a2 = 0;
        slice_accum<T>(vals, A.col, A.off[sl], A.off[sl + 1], p, lane, A.pad, a0, a1, a2);
        row_reduce<T, LPR>(a0, a1, a2);
        const int32_t row = A.rowid[(int64_t)sl * S + r];
        if (q == 0 && row >= 0) store_node(ap, row, a0, a1, a2);
    }
}

__global__ void k_pcg_init(PcgScalars* s, double tol, int32_t max_iter, double delta) {
    s->alpha = 0.0;
    s->beta = 0.0;
    s->rz = 0.0;
    s->rr = s->bb;
    s->tol = tol;
    s->pap = 0.0;
    s->maxr = sqrt(s->bb);
    s->delta = delta;
    s->rr_true = s->bb;
    s->iter = 0;
    s->max_iter = max_iter;
    s->status = 0;
    s->update = 0;
    s->updates = 0;
    s->done = (s->bb == 0.0) ? 1 : 0;  // zero right-hand side: x = 0 (iterative.rs:214-216)
    for (int k = 0; k < 4; ++k) s->ticket[k] = 0;
}

template <typename T>
__global__ void k_norm2(int64_t n, const T* __restrict__ v, double* partials, unsigned int* ticket,
                        double* out) {
    __shared__ double sh[kWarp];
    double loc = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        loc += (double)v[k] * (double)v[k];
    if (publish_partial(loc, partials, ticket, sh)) {
        const double tot = gather_sum(partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            *out = tot;
            *ticket = 0;
        }
    }
}

template <typename T>
__global__ void k_sell_fill(int64_t nslots, const int32_t* __restrict__ src,
                            const double* __restrict__ csr, T* __restrict__ vals) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nslots) return;
    const int64_t g = t / kStepSlots, j = t - g * kStepSlots;
    const int32_t p = src[t];
    const double* m = csr + 9 * (int64_t)(p < 0 ? 0 : p);
#pragma unroll
    for (int k = 0; k < 9; ++k) vals[(g * 9 + k) * kStepSlots + j] = p < 0 ? T(0) : (T)m[k];
}

template <typename T>
__global__ void k_diag_fill(int32_t nb, const int64_t* __restrict__ diag, const double* __restrict__ F,
                            T* __restrict__ D) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
#pragma unroll
    for (int k = 0; k < 9; ++k) D[k * (int64_t)nb + i] = (T)F[9 * diag[i] + k];
}

__global__ void k_cast(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        b[k] = (float)a[k];
}

}  // namespace

#define MAILLE_LPR_SWITCH(lpr, KERNEL, ...)          \
    switch (lpr) {                                   \
        case 1: KERNEL<T, 1><<<__VA_ARGS__; break;   \
        case 2: KERNEL<T, 2><<<__VA_ARGS__; break;   \
        case 4: KERNEL<T, 4><<<__VA_ARGS__; break;   \
        default: KERNEL<T, 8><<<__VA_ARGS__; break;  \
    }

template <typename T>
void launch_spmv(const SellDev& A, const T* vals, const T* p, T* ap, int grid, cudaStream_t st) {
    counted();
    MAILLE_LPR_SWITCH(A.lpr, k_spmv, grid, kThr, 0, st>>>(A, vals, p, ap));
}

void launch_pcg_init(PcgScalars* s, double tol, int32_t max_iter, double delta, cudaStream_t st) {
    counted();
    k_pcg_init<<<1, 1, 0, st>>>(s, tol, max_iter, delta);
}

template <typename T>
void launch_norm2(int64_t n, const T* v, double* partials, unsigned int* ticket, double* out,
                  cudaStream_t st) {
    counted();
    k_norm2<T><<<grid_for(n, kThr, 4), kThr, 0, st>>>(n, v, partials, ticket, out);
}

template <typename T>
void launch_sell_fill(int64_t steps, const int32_t* src, const double* csr, T* vals, cudaStream_t st) {
    counted();
    const int64_t n = steps * kStepSlots;
    k_sell_fill<T><<<(unsigned)((n + kThr - 1) / kThr), kThr, 0, st>>>(n, src, csr, vals);
}

template <typename T>
void launch_diag_fill(int32_t nb, const int64_t* diag, const double* F, T* D, cudaStream_t st) {
    counted();
    k_diag_fill<T><<<(unsigned)((nb + kThr - 1) / kThr), kThr, 0, st>>>(nb, diag, F, D);
}

void launch_cast(int64_t n, const double* a, float* b, cudaStream_t st) {
    counted();
    k_cast<<<grid_for(n, kThr, 32), kThr, 0, st>>>(n, a, b);
}

#define MAILLE_INST(T)                                                                          \
    template void launch_spmv<T>(const SellDev&, const T*, const T*, T*, int, cudaStream_t);   \
    template void launch_norm2<T>(int64_t, const T*, double*, unsigned int*, double*,           \
                                  cudaStream_t);                                                \
    template void launch_sell_fill<T>(int64_t, const int32_t*, const double*, T*, cudaStream_t); \
    template void launch_diag_fill<T>(int32_t, const int64_t*, const double*, T*, cudaStream_t);
MAILLE_INST(float)
MAILLE_INST(double)

}  // namespace maille
