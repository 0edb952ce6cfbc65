// sparse.cu -- SELL 3x3-block SpMV, level-scheduled IC(0) sweeps and the PCG vector kernels.
// Layout and conventions: sparse.cuh. Reductions: reduce.cuh (deterministic).

#include <atomic>
#include <cmath>

#include "reduce.cuh"
#include "sparse.cuh"

namespace maille {

extern std::atomic<long long> g_kernel_launches;

namespace {

constexpr int kThr = 256;
constexpr int kWarp = kThr / 32;
constexpr int kMaxGrid = 148 * 8;

inline int grid_for(int64_t items, int per_block, int cap = kMaxGrid) {
    int64_t g = (items + per_block - 1) / per_block;
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

// acc += this lane's 4 slots of step g: V_b x[col_b] (3x3 blocks)
template <typename T>
__device__ __forceinline__ void step_accum(const T* __restrict__ vals,
                                           const int32_t* __restrict__ col, int64_t g,
                                           const T* __restrict__ x, int lane, T& a0, T& a1, T& a2) {
    const int4 c4 = __ldg(reinterpret_cast<const int4*>(col + g * kStepSlots + 4 * lane));
    const T* V = vals + g * 9 * kStepSlots + 4 * lane;
    T v[9][4];
#pragma unroll
    for (int k = 0; k < 9; ++k) load4(V + k * kStepSlots, v[k]);
    const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        T x0, x1, x2;
        node3(x, cc[j], x0, x1, x2);
        a0 += v[0][j] * x0 + v[1][j] * x1 + v[2][j] * x2;
        a1 += v[3][j] * x0 + v[4][j] * x1 + v[5][j] * x2;
        a2 += v[6][j] * x0 + v[7][j] * x1 + v[8][j] * x2;
    }
}

// acc += sum over the slice steps [g0, g1) of this lane's slots
template <typename T>
__device__ __forceinline__ void slice_accum(const T* __restrict__ vals,
                                            const int32_t* __restrict__ col, int64_t g0, int64_t g1,
                                            const T* __restrict__ x, int lane, T& a0, T& a1, T& a2) {
#pragma unroll 2
    for (int64_t g = g0; g < g1; ++g) step_accum<T>(vals, col, g, x, lane, a0, a1, a2);
}

// Slice sum split across the kSweepWarps warps of a block: warp w takes steps g0 + w,
// g0 + w + kSweepWarps, ...; the partial sums meet in shared memory and warp 0 returns the total
// (the other warps return 0). Summation order is fixed, so results are deterministic.
constexpr int kSweepWarps = 8;
template <typename T>
__device__ __forceinline__ void slice_accum_cta(const T* __restrict__ vals,
                                                const int32_t* __restrict__ col, int64_t g0,
                                                int64_t g1, const T* __restrict__ x, T (*red)[32][3],
                                                T& a0, T& a1, T& a2) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    a0 = 0;
    a1 = 0;
    a2 = 0;
    for (int64_t g = g0 + w; g < g1; g += kSweepWarps) step_accum<T>(vals, col, g, x, lane, a0, a1, a2);
    if (w > 0) {
        red[w - 1][lane][0] = a0;
        red[w - 1][lane][1] = a1;
        red[w - 1][lane][2] = a2;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < kSweepWarps - 1; ++k) {
            a0 += red[k][lane][0];
            a1 += red[k][lane][1];
            a2 += red[k][lane][2];
        }
    }
    __syncthreads();
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

// ap = K p (Csr::multiply, iterative.rs:131-142, as a gather on the full symmetric pattern),
// p . ap reduced; the last block sets alpha = rz / (p . ap) and counts the iteration, or flags
// SINGULAR on curvature <= 0 / NaN (iterative.rs:223-228). `standalone` launches (timing) skip
// the done check and the scalar update.
template <typename T, int LPR>
__global__ void __launch_bounds__(kThr) k_spmv(SellDev A, const T* __restrict__ vals,
                                                const T* __restrict__ p, T* __restrict__ ap,
                                                PcgScalars* s, double* partials, int standalone) {
    __shared__ double sh[kWarp];
    if (!standalone && s->done) return;
    const int lane = threadIdx.x & 31, r = lane / LPR, q = lane % LPR;
    constexpr int S = 32 / LPR;
    double loc = 0.0;
    for (int32_t sl = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); sl < A.nslices;
         sl += (int32_t)((gridDim.x * blockDim.x) >> 5)) {
        T a0 = 0, a1 = 0, a2 = 0;
        slice_accum<T>(vals, A.col, A.off[sl], A.off[sl + 1], p, lane, a0, a1, a2);
        row_reduce<T, LPR>(a0, a1, a2);
        const int32_t row = A.rowid[(int64_t)sl * S + r];
        if (q == 0 && row >= 0) {
            store_node(ap, row, a0, a1, a2);
            T p0, p1, p2;
            node3(p, row, p0, p1, p2);
            loc += (double)p0 * (double)a0 + (double)p1 * (double)a1 + (double)p2 * (double)a2;
        }
    }
    if (standalone) return;
    if (publish_partial(loc, partials, &s->ticket[0], sh)) {
        const double pap = gather_sum(partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            s->pap = pap;
            s->iter += 1;
            if (isnan(pap) || pap <= 0.0) {
                s->status = 1;
                s->done = 1;
            } else {
                s->alpha = s->rz / pap;
            }
            s->ticket[0] = 0;
        }
    }
}

// x += alpha p, r -= alpha ap (iterative.rs:229-232) with ||r||^2. Plain form: the last block
// applies the reference's stopping test ||r|| <= tol ||b|| (iterative.rs:233) and the cap.
// Mixed form: it raises `update` (a reliable update of x and r in FP64) when the iterated
// residual fell by `delta` since the last update, claims convergence, or the cap is reached.
template <typename T>
__global__ void __launch_bounds__(kThr) k_axpy(int32_t nb, T* __restrict__ x, T* __restrict__ r,
                                                const T* __restrict__ p, const T* __restrict__ ap,
                                                PcgScalars* s, double* partials, int mixed) {
    __shared__ double sh[kWarp];
    if (s->done) return;
    const double alpha = s->alpha;
    double loc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb;
         i += (int64_t)gridDim.x * blockDim.x) {
        F4 xv = ld4(x, i), rv = ld4(r, i);
        const F4 pv = ld4(p, i), av = ld4(ap, i);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            xv.v[c] = (double)(T)(xv.v[c] + alpha * pv.v[c]);
            rv.v[c] = (double)(T)(rv.v[c] - alpha * av.v[c]);
            loc += rv.v[c] * rv.v[c];
        }
        st4(x, i, xv);
        st4(r, i, rv);
    }
    if (publish_partial(loc, partials, &s->ticket[1], sh)) {
        const double rr = gather_sum(partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            s->rr = rr;
            s->ticket[1] = 0;
            const bool small = sqrt(rr) <= s->tol * sqrt(s->bb);
            if (!mixed) {
                if (small) {
                    s->done = 1;
                } else if (s->iter >= s->max_iter) {
                    s->done = 1;
                    s->status = 2;
                }
            } else {
                s->update = (small || sqrt(rr) < s->delta * s->maxr || s->iter >= s->max_iter) ? 1 : 0;
            }
        }
    }
}

// reliable update, part 1: x64 += x32, x32 = 0
__global__ void k_upd_x(int32_t nb, double* __restrict__ x64, float* __restrict__ x32, PcgScalars* s) {
    if (s->done || !s->update) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb;
         i += (int64_t)gridDim.x * blockDim.x) {
        F4 a = ld4(x64, i);
        const F4 d = ld4(x32, i);
#pragma unroll
        for (int c = 0; c < 4; ++c) a.v[c] += d.v[c];
        st4(x64, i, a);
        st4(x32, i, F4{{0.0, 0.0, 0.0, 0.0}});
    }
}

// reliable update, part 2: the true residual r64 = b - K64 x64 against the FP64 matrix, its norm
// and the convergence test on it.
template <int LPR>
__global__ void __launch_bounds__(kThr) k_upd_r(SellDev A, const double* __restrict__ vals,
                                                 const double* __restrict__ b,
                                                 const double* __restrict__ x64,
                                                 double* __restrict__ r64, PcgScalars* s,
                                                 double* partials) {
    __shared__ double sh[kWarp];
    if (s->done || !s->update) return;
    const int lane = threadIdx.x & 31;
    double loc = 0.0;
    for (int32_t sl = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); sl < A.nslices;
         sl += (int32_t)((gridDim.x * blockDim.x) >> 5)) {
        double a0 = 0, a1 = 0, a2 = 0;
        slice_accum<double>(vals, A.col, A.off[sl], A.off[sl + 1], x64, lane, a0, a1, a2);
        row_reduce<double, LPR>(a0, a1, a2);
        const int32_t row = A.rowid[(int64_t)sl * (32 / LPR) + lane / LPR];
        if (lane % LPR == 0 && row >= 0) {
            const double q0 = b[4 * (int64_t)row] - a0, q1 = b[4 * (int64_t)row + 1] - a1,
                         q2 = b[4 * (int64_t)row + 2] - a2;
            store_node(r64, row, q0, q1, q2);
            loc += q0 * q0 + q1 * q1 + q2 * q2;
        }
    }
    if (publish_partial(loc, partials, &s->ticket[3], sh)) {
        const double rr = gather_sum(partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            s->rr_true = rr;
            s->maxr = sqrt(rr);
            s->updates += 1;
            s->ticket[3] = 0;
            if (sqrt(rr) <= s->tol * sqrt(s->bb)) {
                s->done = 1;
            } else if (s->iter >= s->max_iter) {
                s->done = 1;
                s->status = 2;
            }
        }
    }
}

// reliable update, part 3: the FP32 recurrence restarts from the true residual
__global__ void k_upd_cast(int32_t nb, const double* __restrict__ r64, float* __restrict__ r32,
                           PcgScalars* s) {
    if (s->done || !s->update) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb;
         i += (int64_t)gridDim.x * blockDim.x)
        st4(r32, i, ld4(r64, i));
}

// One level of the forward sweep y_I = L_II^-1 (r_I - sum_{J<I} L_IJ y_J) (Csr::precondition,
// iterative.rs:175-179, block form; D_I = L_II^-1 stored as 9 planes of nb entries). One block of
// kSweepWarps warps per slice: the warps split the slice's steps, so a level with few slices still
// keeps every SM busy.
template <typename T, int LPR>
__global__ void __launch_bounds__(kSweepWarps * 32) k_fwd(SellDev Lm, int32_t s0, int32_t s1,
                                                          const T* __restrict__ vals,
                                                          const T* __restrict__ D, int32_t nb,
                                                          const T* __restrict__ r, T* y,
                                                          const PcgScalars* s) {
    __shared__ T red[kSweepWarps - 1][32][3];
    if (s->done) return;
    const int lane = threadIdx.x & 31, rr = lane / LPR, q = lane % LPR;
    constexpr int S = 32 / LPR;
    for (int32_t sl = s0 + (int32_t)blockIdx.x; sl < s1; sl += (int32_t)gridDim.x) {
        T a0, a1, a2;
        slice_accum_cta<T>(vals, Lm.col, Lm.off[sl], Lm.off[sl + 1], y, red, a0, a1, a2);
        if (threadIdx.x < 32) {
            row_reduce<T, LPR>(a0, a1, a2);
            const int32_t row = Lm.rowid[(int64_t)sl * S + rr];
            if (q == 0 && row >= 0) {
                T r0, r1, r2;
                node3(r, row, r0, r1, r2);
                const T u0 = r0 - a0, u1 = r1 - a1, u2 = r2 - a2;
                const T* d = D + row;
                const T y0 = d[0] * u0;
                const T y1 = d[3 * (int64_t)nb] * u0 + d[4 * (int64_t)nb] * u1;
                const T y2 = d[6 * (int64_t)nb] * u0 + d[7 * (int64_t)nb] * u1 + d[8 * (int64_t)nb] * u2;
                store_node(y, row, y0, y1, y2);
            }
        }
    }
}

// One level of the backward sweep z_I = L_II^-T (y_I - sum_{J>I} L_JI^T z_J), in place over y
// (Csr::precondition, iterative.rs:180-186, as a gather on the stored upper blocks L_JI^T), with
// r . z partials; the last launch (level 0) sets beta = rz_new / rz, rz = rz_new
// (iterative.rs:237-239). One block per slice, as in the forward sweep.
template <typename T, int LPR>
__global__ void __launch_bounds__(kSweepWarps * 32) k_bwd(SellDev Um, int32_t s0, int32_t s1,
                                                          int level, int nlevels,
                                                          const T* __restrict__ vals,
                                                          const T* __restrict__ D, int32_t nb,
                                                          const T* __restrict__ r, T* z,
                                                          PcgScalars* s, double* partials,
                                                          double* lvl_total) {
    __shared__ T red[kSweepWarps - 1][32][3];
    __shared__ double sh[kSweepWarps];
    if (s->done) return;
    const int lane = threadIdx.x & 31, rr = lane / LPR, q = lane % LPR;
    constexpr int S = 32 / LPR;
    double loc = 0.0;
    for (int32_t sl = s0 + (int32_t)blockIdx.x; sl < s1; sl += (int32_t)gridDim.x) {
        T a0, a1, a2;
        slice_accum_cta<T>(vals, Um.col, Um.off[sl], Um.off[sl + 1], z, red, a0, a1, a2);
        if (threadIdx.x < 32) {
            row_reduce<T, LPR>(a0, a1, a2);
            const int32_t row = Um.rowid[(int64_t)sl * S + rr];
            if (q == 0 && row >= 0) {
                T y0, y1, y2;
                node3_rw(z, row, y0, y1, y2);
                const T u0 = y0 - a0, u1 = y1 - a1, u2 = y2 - a2;
                const T* d = D + row;
                const T z0 = d[0] * u0 + d[3 * (int64_t)nb] * u1 + d[6 * (int64_t)nb] * u2;
                const T z1 = d[4 * (int64_t)nb] * u1 + d[7 * (int64_t)nb] * u2;
                const T z2 = d[8 * (int64_t)nb] * u2;
                store_node(z, row, z0, z1, z2);
                T r0, r1, r2;
                node3(r, row, r0, r1, r2);
                loc += (double)r0 * (double)z0 + (double)r1 * (double)z1 + (double)r2 * (double)z2;
            }
        }
    }
    if (publish_partial(loc, partials, &s->ticket[2], sh)) {
        const double tot = gather_sum(partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            lvl_total[level] = tot;
            s->ticket[2] = 0;
        }
        if (level == 0) {
            const double rz = gather_sum(lvl_total, nlevels, sh);
            if (threadIdx.x == 0) {
                s->beta = (s->iter == 0) ? 0.0 : rz / s->rz;
                s->rz = rz;
            }
        }
    }
}

// p = z + beta p (iterative.rs:240-242)
template <typename T>
__global__ void k_pupdate(int32_t nb, const T* __restrict__ z, T* __restrict__ p, PcgScalars* s) {
    if (s->done) return;
    const double beta = s->beta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb;
         i += (int64_t)gridDim.x * blockDim.x) {
        const F4 zv = ld4(z, i);
        F4 pv = ld4(p, i);
#pragma unroll
        for (int c = 0; c < 4; ++c) pv.v[c] = zv.v[c] + beta * pv.v[c];
        st4(p, i, pv);
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

template <int LPR>
__global__ void __launch_bounds__(kThr) k_residual64(SellDev A, const double* __restrict__ vals,
                                                      const double* __restrict__ b,
                                                      const double* __restrict__ u,
                                                      double* __restrict__ r, double* partials,
                                                      unsigned int* ticket, double* out) {
    __shared__ double sh[kWarp];
    const int lane = threadIdx.x & 31;
    double loc = 0.0;
    for (int32_t sl = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); sl < A.nslices;
         sl += (int32_t)((gridDim.x * blockDim.x) >> 5)) {
        double a0 = 0, a1 = 0, a2 = 0;
        slice_accum<double>(vals, A.col, A.off[sl], A.off[sl + 1], u, lane, a0, a1, a2);
        row_reduce<double, LPR>(a0, a1, a2);
        const int32_t row = A.rowid[(int64_t)sl * (32 / LPR) + lane / LPR];
        if (lane % LPR == 0 && row >= 0) {
            const double q0 = b[4 * (int64_t)row] - a0, q1 = b[4 * (int64_t)row + 1] - a1,
                         q2 = b[4 * (int64_t)row + 2] - a2;
            store_node(r, row, q0, q1, q2);
            loc += q0 * q0 + q1 * q1 + q2 * q2;
        }
    }
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
void launch_spmv(const SellDev& A, const T* vals, const T* p, T* ap, PcgScalars* s,
                 double* partials, int grid, bool standalone, cudaStream_t st) {
    counted();
    MAILLE_LPR_SWITCH(A.lpr, k_spmv, grid, kThr, 0, st>>>(A, vals, p, ap, s, partials, standalone ? 1 : 0));
}

template <typename T>
void launch_axpy(int32_t nb, T* x, T* r, const T* p, const T* ap, PcgScalars* s, double* partials,
                 bool mixed, cudaStream_t st) {
    counted();
    k_axpy<T><<<grid_for(nb, kThr, 148 * 16), kThr, 0, st>>>(nb, x, r, p, ap, s, partials, mixed ? 1 : 0);
}

void launch_upd_x(int32_t nb, double* x64, float* x32, PcgScalars* s, cudaStream_t st) {
    counted();
    k_upd_x<<<grid_for(nb, kThr, 148 * 16), kThr, 0, st>>>(nb, x64, x32, s);
}

void launch_upd_r(const SellDev& A, const double* vals, const double* b, const double* x64,
                  double* r64, PcgScalars* s, double* partials, int grid, cudaStream_t st) {
    counted();
    using T = double;
    (void)sizeof(T);
    switch (A.lpr) {
        case 1: k_upd_r<1><<<grid, kThr, 0, st>>>(A, vals, b, x64, r64, s, partials); break;
        case 2: k_upd_r<2><<<grid, kThr, 0, st>>>(A, vals, b, x64, r64, s, partials); break;
        case 4: k_upd_r<4><<<grid, kThr, 0, st>>>(A, vals, b, x64, r64, s, partials); break;
        default: k_upd_r<8><<<grid, kThr, 0, st>>>(A, vals, b, x64, r64, s, partials); break;
    }
}

void launch_upd_cast(int32_t nb, const double* r64, float* r32, PcgScalars* s, cudaStream_t st) {
    counted();
    k_upd_cast<<<grid_for(nb, kThr, 148 * 16), kThr, 0, st>>>(nb, r64, r32, s);
}

template <typename T>
void launch_fwd(const SellDev& L, int32_t s0, int32_t s1, const T* vals, const T* D, int32_t nb,
                const T* r, T* y, PcgScalars* s, cudaStream_t st) {
    counted();
    const int grid = grid_for(s1 - s0, 1, 148 * 16);
    MAILLE_LPR_SWITCH(L.lpr, k_fwd, grid, kSweepWarps * 32, 0, st>>>(L, s0, s1, vals, D, nb, r, y, s));
}

template <typename T>
void launch_bwd(const SellDev& U, int32_t s0, int32_t s1, int level, int nlevels, const T* vals,
                const T* D, int32_t nb, const T* r, T* z, PcgScalars* s, double* partials,
                double* lvl_total, cudaStream_t st) {
    counted();
    const int grid = grid_for(s1 - s0, 1, 148 * 16);
    MAILLE_LPR_SWITCH(U.lpr, k_bwd, grid, kSweepWarps * 32, 0, st>>>(U, s0, s1, level, nlevels, vals, D, nb, r, z, s, partials, lvl_total));
}

template <typename T>
void launch_pupdate(int32_t nb, const T* z, T* p, PcgScalars* s, cudaStream_t st) {
    counted();
    k_pupdate<T><<<grid_for(nb, kThr, 148 * 16), kThr, 0, st>>>(nb, z, p, s);
}

void launch_pcg_init(PcgScalars* s, double tol, int32_t max_iter, double delta, cudaStream_t st) {
    counted();
    k_pcg_init<<<1, 1, 0, st>>>(s, tol, max_iter, delta);
}

template <typename T>
void launch_norm2(int64_t n, const T* v, double* partials, unsigned int* ticket, double* out,
                  cudaStream_t st) {
    counted();
    k_norm2<T><<<grid_for(n, kThr, 148 * 4), kThr, 0, st>>>(n, v, partials, ticket, out);
}

void launch_residual64(const SellDev& A, const double* vals, const double* b, const double* u,
                       double* r, double* partials, unsigned int* ticket, double* out, int grid,
                       cudaStream_t st) {
    counted();
    switch (A.lpr) {
        case 1: k_residual64<1><<<grid, kThr, 0, st>>>(A, vals, b, u, r, partials, ticket, out); break;
        case 2: k_residual64<2><<<grid, kThr, 0, st>>>(A, vals, b, u, r, partials, ticket, out); break;
        case 4: k_residual64<4><<<grid, kThr, 0, st>>>(A, vals, b, u, r, partials, ticket, out); break;
        default: k_residual64<8><<<grid, kThr, 0, st>>>(A, vals, b, u, r, partials, ticket, out); break;
    }
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
    k_cast<<<grid_for(n, kThr, 148 * 32), kThr, 0, st>>>(n, a, b);
}

#define MAILLE_INST(T)                                                                          \
    template void launch_spmv<T>(const SellDev&, const T*, const T*, T*, PcgScalars*, double*,  \
                                 int, bool, cudaStream_t);                                      \
    template void launch_axpy<T>(int32_t, T*, T*, const T*, const T*, PcgScalars*, double*,     \
                                 bool, cudaStream_t);                                           \
    template void launch_fwd<T>(const SellDev&, int32_t, int32_t, const T*, const T*, int32_t, \
                                const T*, T*, PcgScalars*, cudaStream_t);                       \
    template void launch_bwd<T>(const SellDev&, int32_t, int32_t, int, int, const T*, const T*, \
                                int32_t, const T*, T*, PcgScalars*, double*, double*,          \
                                cudaStream_t);                                                  \
    template void launch_pupdate<T>(int32_t, const T*, T*, PcgScalars*, cudaStream_t);          \
    template void launch_norm2<T>(int64_t, const T*, double*, unsigned int*, double*,           \
                                  cudaStream_t);                                                \
    template void launch_sell_fill<T>(int64_t, const int32_t*, const double*, T*, cudaStream_t); \
    template void launch_diag_fill<T>(int32_t, const int64_t*, const double*, T*, cudaStream_t);
MAILLE_INST(float)
MAILLE_INST(double)

}  // namespace maille
